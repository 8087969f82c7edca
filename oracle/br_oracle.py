"""CPU restatement of the regrid step's tagging and Berger-Rigoutsos
clustering (numpy / plain Python).

TEST INFRASTRUCTURE ONLY: the checker for the device tagging and clustering
(samrai_b200 fac_tag_gradient / fac_cluster_tags); pinned to the reference's
own routines by tests/golden/ref_br_*.npz (oracle/_ref/br_ref_driver).

* adaption_estimate: AdaptivePoisson::computeAdaptionEstimate
  (source/test/FAC_adaptive/AdaptivePoisson.C:622-720): the largest absolute
  second difference of u along the axes, and half of it along the face
  diagonals, per cell, evaluated as (u(+) + u(-)) - 2 u(0).
* tag = estimate > threshold (AdaptivePoisson.C:517-527).
* cluster: BergerRigoutsos / BergerRigoutsosNode on one process
  (mesh/BergerRigoutsosNode.C): per node the tag histogram along each axis
  (makeLocalTagHistogram, :1186-1241), the minimal bounding box
  (computeMinimalBoundingBoxForTags, :1251-1318), acceptance by efficiency
  or by size, else a cut at a zero swath of the histogram nearest the
  middle (findZeroCutSwath, :1636-1700) along the directions of largest cut
  margin first, else at the strongest inflection of the histogram's
  Laplacian (cutAtInflection, :1718-1812) along the longest direction(s);
  children run depth first and are recombined into the parent when both
  were accepted and their cells make up at least combine_efficiency of the
  parent's (runChildren_check, :719-790).  Defaults of the reference: no
  maximum box size, DEV_max_inflection_cut_from_center 1,
  DEV_inflection_cut_threshold_ar 0, DEV_min_box_size_from_cutting 0.
"""
from __future__ import annotations

import numpy as np


def adaption_estimate(u_ghosted: np.ndarray, dim: int) -> np.ndarray:
    """Estimate on the interior of one patch from its ghost-1 array (numpy
    order z, y, x in 3-D, y, x in 2-D)."""
    c = u_ghosted
    if dim == 2:
        ctr = c[1:-1, 1:-1]

        def sh(dx, dy):
            return c[1 + dy:c.shape[0] - 1 + dy, 1 + dx:c.shape[1] - 1 + dx]

        def d2(p, m):
            return np.abs((sh(*p) + sh(*m)) - 2 * ctr)
        est0 = d2((1, 0), (-1, 0))
        est1 = d2((0, 1), (0, -1))
        est2 = 0.5 * d2((1, 1), (-1, -1))
        est3 = 0.5 * d2((1, -1), (-1, 1))
        return np.maximum(np.maximum(est0, est1), np.maximum(est2, est3))
    ctr = c[1:-1, 1:-1, 1:-1]

    def sh3(dx, dy, dz):
        return c[1 + dz:c.shape[0] - 1 + dz, 1 + dy:c.shape[1] - 1 + dy,
                 1 + dx:c.shape[2] - 1 + dx]

    def d3(p, m):
        return np.abs((sh3(*p) + sh3(*m)) - 2 * ctr)
    est0 = d3((1, 0, 0), (-1, 0, 0))
    est1 = d3((0, 1, 0), (0, -1, 0))
    est2 = d3((0, 0, 1), (0, 0, -1))
    est3 = 0.5 * d3((0, 1, 1), (0, -1, -1))
    est4 = 0.5 * d3((0, 1, -1), (0, -1, 1))
    est5 = 0.5 * d3((1, 0, 1), (-1, 0, -1))
    est6 = 0.5 * d3((1, 0, -1), (-1, 0, 1))
    est7 = 0.5 * d3((1, 1, 0), (-1, -1, 0))
    est8 = 0.5 * d3((1, -1, 0), (-1, 1, 0))
    esta = np.maximum(est0, est1)
    estb = np.maximum(est2, est3)
    estc = np.maximum(est4, est5)
    estd = np.maximum(est6, est7)
    este = np.maximum(esta, estb)
    estf = np.maximum(estc, estd)
    estg = np.maximum(este, estf)
    return np.maximum(estg, est8)


def cdiv(a: int, b: int) -> int:
    """C integer division (toward zero)."""
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


class Clusterer:
    """Berger-Rigoutsos over a dense tag array covering [lo, lo + shape)."""

    def __init__(self, tags: np.ndarray, lo, dim: int, min_box, max_box=None,
                 efficiency=0.8, combine=0.8):
        self.t = tags.astype(np.int64)
        self.lo = [int(x) for x in lo]
        self.dim = dim
        self.min_box = [int(x) for x in min_box[:dim]]
        big = np.iinfo(np.int32).max
        self.max_box = [int(x) if x and x > 0 else big for x in (max_box or [0] * dim)[:dim]]
        self.eff = float(efficiency)
        self.comb = float(combine)

    def _histogram(self, blo, bhi):
        d = self.dim
        # numpy axis of index direction a: 3-D (z, y, x), 2-D (y, x)
        sl = tuple(slice(blo[a] - self.lo[a], bhi[a] - self.lo[a] + 1) for a in reversed(range(d)))
        sub = self.t[sl]
        h = []
        for a in range(d):
            ax = d - 1 - a
            other = tuple(x for x in range(d) if x != ax)
            h.append([int(v) for v in sub.sum(axis=other)])
        return h

    def _shrink(self, blo, bhi, h):
        blo, bhi = list(blo), list(bhi)
        for a in range(self.dim):
            size = bhi[a] - blo[a] + 1
            b, e = 0, len(h[a]) - 1
            while h[a][b] == 0 and size > self.min_box[a]:
                blo[a] += 1
                b += 1
                size -= 1
            while h[a][e] == 0 and size > self.min_box[a]:
                bhi[a] -= 1
                e -= 1
                size -= 1
            h[a] = h[a][b:e + 1]
        return blo, bhi, h

    def _zero_cut(self, blo, bhi, h, a):
        lo, hi = blo[a], bhi[a]
        lim_lo, lim_hi = lo + self.min_box[a], hi - self.min_box[a]
        cl = ch = cdiv(lo + hi, 2)
        hist = h[a]
        while cl >= lim_lo and ch <= lim_hi:
            if hist[cl - lo] == 0:
                ch = cl
                while cl > lim_lo and hist[cl - lo - 1] == 0:
                    cl -= 1
                return cl, ch
            if hist[ch - lo] == 0:
                cl = ch
                while ch < lim_hi and hist[ch - lo + 1] == 0:
                    ch += 1
                return cl, ch
            cl -= 1
            ch += 1
        return None

    def _inflection(self, blo, h, a):
        hist = h[a]
        n = len(hist)
        if n < 4:
            cut = 1
            for i in range(2, n):
                if abs(hist[cut] - hist[cut - 1]) < abs(hist[i] - hist[i - 1]):
                    cut = i
            return cut + blo[a], 0
        mbs = max(self.min_box[a], 0)
        box_lo, box_hi = 0, n - 1
        max_dist = int(1.0 * n / 2)
        mid = cdiv(box_lo + box_hi + 1, 2)
        lim_lo = max(box_lo + mbs, mid - max_dist)
        lim_hi = min(box_hi - mbs + 1, mid + max_dist)
        cut = mid
        infl = abs((hist[cut - 1] - 2 * hist[cut] + hist[cut + 1]) -
                   (hist[cut - 2] - 2 * hist[cut - 1] + hist[cut]))
        cl, ch = mid - 1, mid + 1
        while cl > lim_lo or ch < lim_hi:
            for c, ok in ((cl, cl > lim_lo), (ch, ch < lim_hi)):
                if not ok:
                    continue
                la = hist[c - 1] - 2 * hist[c] + hist[c + 1]
                lb = hist[c - 2] - 2 * hist[c - 1] + hist[c]
                if la * lb <= 0:
                    t = abs(la - lb)
                    if t > infl:
                        cut, infl = c, t
            cl -= 1
            ch += 1
        return cut + blo[a], infl

    def _node(self, blo, bhi, root):
        """Returns (accepted, box after shrink, boxes of the subtree)."""
        d = self.dim
        h = self._histogram(blo, bhi)
        blo, bhi, h = self._shrink(blo, bhi, h)
        dims = [bhi[a] - blo[a] + 1 for a in range(d)]
        size = int(np.prod(dims))
        state = None
        if all(dims[a] - self.max_box[a] <= 0 for a in range(d)):
            ntag = sum(h[0])
            eff = 1.0 if size == 0 else ntag / size
            if eff >= self.eff:
                state = "accept"
            elif ntag == 0:
                state = "notag"
        margin = [dims[a] - 2 * self.min_box[a] for a in range(d)]
        # IntVector's < holds when it holds in every direction: the box is
        # kept whole only when no direction can be cut
        if state is None and all(m < 0 for m in margin):
            state = "accept"
        if state == "accept":
            return True, (blo, bhi), [(tuple(blo), tuple(bhi))]
        if state == "notag":
            return False, (blo, bhi), []
        order = list(range(d))
        for d0 in range(d - 1):
            for d1 in range(d0 + 1, d):
                if margin[order[d0]] < margin[order[d1]]:
                    order[d0], order[d1] = order[d1], order[d0]
        lft_hi, rht_lo = list(bhi), list(blo)
        cut_dir = 0
        found = False
        for k in range(d):
            cut_dir = order[k]
            if margin[cut_dir] < 0:
                continue
            z = self._zero_cut(blo, bhi, h, cut_dir)
            if z is not None:
                lft_hi[cut_dir] = z[0] - 1
                rht_lo[cut_dir] = z[1] + 1
                found = True
                break
        if not found:
            leave = dims[order[0]] - 1
            infl, cut_pt = -1, None
            for a in range(d):
                if margin[a] < 0 or dims[a] <= leave:
                    continue
                cp, ti = self._inflection(blo, h, a)
                if infl < ti or (infl == ti and margin[a] > margin[cut_dir]):
                    cut_dir, cut_pt, infl = a, cp, ti
            lft_hi[cut_dir] = cut_pt - 1
            rht_lo[cut_dir] = cut_pt
        la, lbox, lout = self._node(list(blo), lft_hi, False)
        ra, rbox, rout = self._node(rht_lo, list(bhi), False)
        lsize = int(np.prod([lbox[1][a] - lbox[0][a] + 1 for a in range(d)]))
        rsize = int(np.prod([rbox[1][a] - rbox[0][a] + 1 for a in range(d)]))
        if (la and ra and all(dims[a] <= self.max_box[a] for a in range(d)) and
                (lsize + rsize) / size >= self.comb):
            return True, (blo, bhi), [(tuple(blo), tuple(bhi))]
        return False, (blo, bhi), lout + rout

    def cluster(self, bound_boxes):
        """Boxes ((lo), (hi)) covering the tags inside each bound box."""
        out = []
        for b in bound_boxes:
            blo, bhi = [int(x) for x in b[:self.dim]], [int(x) for x in b[3:3 + self.dim]]
            out += self._node(blo, bhi, True)[2]
        return out
