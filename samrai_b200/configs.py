"""Synthetic, seeded FAC problems (hierarchies, right-hand sides, coefficients).

The reference's own drivers build hierarchies with GriddingAlgorithm
(source/test/FAC_staticrefinement/main.C, FACPoisson.C:244-300) or read them
from input files; the five benchmark configurations here are built directly
from boxes, as the reference's static-refinement test does with its
``refine_boxes`` input.  Every index box is aligned to the refinement ratio
and every refined level is properly nested in its parent with a buffer of at
least one parent cell, as SAMRAI's gridding guarantees.

A :class:`Problem` is pure data (numpy arrays); the solver (``samrai_b200.fac``)
and the CPU oracle consume the same description.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np


@dataclasses.dataclass
class Level:
    ratio: tuple          # refinement ratio to the next coarser level (1s on level 0)
    boxes: np.ndarray     # (npatch, 6) int32: lo0 lo1 lo2 hi0 hi1 hi2


@dataclasses.dataclass
class Problem:
    dim: int
    n0: tuple             # level-0 cells per axis (domain is [0, n0-1])
    xlo: tuple
    xup: tuple
    levels: List[Level]
    # Poisson specification: div(D grad u) + C u = f
    d_variable: bool = False
    d_const: float = 1.0
    c_kind: int = 0       # 0 zero, 1 constant, 2 variable
    c_const: float = 0.0
    # per level canonical arrays (filled by the builders below)
    f: List[np.ndarray] = dataclasses.field(default_factory=list)
    u0: List[np.ndarray] = dataclasses.field(default_factory=list)
    d: List[np.ndarray] = dataclasses.field(default_factory=list)  # side data
    c: List[np.ndarray] = dataclasses.field(default_factory=list)
    name: str = ""

    @property
    def nlev(self):
        return len(self.levels)

    def ratio_to_zero(self, ln):
        r = np.ones(3, dtype=np.int64)
        for l in range(1, ln + 1):
            r *= np.asarray(self.levels[l].ratio, dtype=np.int64)
        return r

    def dx(self, ln):
        rz = self.ratio_to_zero(ln)
        out = []
        for a in range(3):
            if a < self.dim:
                dx0 = (self.xup[a] - self.xlo[a]) / float(self.n0[a])
                out.append(dx0 / float(rz[a]))
            else:
                out.append(1.0)
        return out

    def domain(self, ln):
        rz = self.ratio_to_zero(ln)
        hi = [int(self.n0[a] * rz[a] - 1) if a < self.dim else 0 for a in range(3)]
        return [0, 0, 0], hi

    def num_cells(self):
        n = 0
        for L in self.levels:
            b = L.boxes
            n += int(np.prod(b[:, 3:] - b[:, :3] + 1, axis=1).sum())
        return n

    def num_patches(self):
        return sum(len(L.boxes) for L in self.levels)


# ---------------------------------------------------------------------------
# layout helpers (canonical layout = concatenated ghosted patch arrays)
# ---------------------------------------------------------------------------

def _ghost_vec(dim, g):
    return np.array([g, g, g if dim == 3 else 0])


def cell_shape(dim, box, g):
    gv = _ghost_vec(dim, g)
    lo = np.asarray(box[:3]) - gv
    hi = np.asarray(box[3:]) + gv
    return lo, (hi - lo + 1)


def field_size(prob: Problem, ln: int, g: int) -> int:
    n = 0
    for b in prob.levels[ln].boxes:
        _, ext = cell_shape(prob.dim, b, g)
        n += int(np.prod(ext))
    return n


def side_size(prob: Problem, ln: int) -> int:
    n = 0
    for b in prob.levels[ln].boxes:
        ext = b[3:] - b[:3] + 1
        for a in range(prob.dim):
            e = ext.copy()
            e[a] += 1
            n += int(np.prod(e))
    return n


def patch_views(prob: Problem, ln: int, arr: np.ndarray, g: int):
    """Yield (box, lo, view[z,y,x]) for each patch of a canonical cell array."""
    off = 0
    for b in prob.levels[ln].boxes:
        lo, ext = cell_shape(prob.dim, b, g)
        n = int(np.prod(ext))
        v = arr[off:off + n].reshape(ext[2], ext[1], ext[0])
        yield b, lo, v
        off += n


def cell_centers(prob: Problem, ln: int, box, g=0):
    dx = prob.dx(ln)
    lo, ext = cell_shape(prob.dim, box, g)
    xs = [prob.xlo[a] + (np.arange(lo[a], lo[a] + ext[a]) + 0.5) * dx[a]
          if a < prob.dim else np.zeros(1) for a in range(3)]
    Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
    return X, Y, Z


def fill_cell_field(prob: Problem, ln: int, g: int, fn) -> np.ndarray:
    out = np.zeros(field_size(prob, ln, g))
    for b, lo, v in patch_views(prob, ln, out, g):
        X, Y, Z = cell_centers(prob, ln, b, g)
        v[...] = fn(X, Y, Z)
    return out


def fill_side_field(prob: Problem, ln: int, fn) -> np.ndarray:
    """Side (face-centred) data, evaluated at face centres
    (as PoissonGaussianDiffcoefSolution.C:178-216 sets D)."""
    dx = prob.dx(ln)
    out = np.zeros(side_size(prob, ln))
    off = 0
    for b in prob.levels[ln].boxes:
        for a in range(prob.dim):
            lo = b[:3].copy()
            hi = b[3:].copy()
            hi[a] += 1
            ext = hi - lo + 1
            xs = []
            for t in range(3):
                idx = np.arange(lo[t], hi[t] + 1, dtype=np.float64)
                if t >= prob.dim:
                    xs.append(np.zeros(1))
                elif t == a:
                    xs.append(prob.xlo[t] + idx * dx[t])
                else:
                    xs.append(prob.xlo[t] + (idx + 0.5) * dx[t])
            n = int(np.prod(ext))
            if hasattr(fn, "grid"):
                out[off:off + n] = fn.grid(xs[0], xs[1], xs[2]).reshape(-1)
            else:
                Z, Y, X = np.meshgrid(xs[2], xs[1], xs[0], indexing="ij")
                out[off:off + n] = fn(X, Y, Z).reshape(-1)
            off += n
    return out


# ---------------------------------------------------------------------------
# box algebra for the generators
# ---------------------------------------------------------------------------

def _mask_to_boxes(mask: np.ndarray, block: int, max_side_blocks: int, dim: int):
    """Greedy decomposition of a block mask (z, y, x) into disjoint boxes of
    at most ``max_side_blocks`` blocks per side.  Returns (n, 6) boxes in
    cell units."""
    m = mask.copy()
    boxes = []
    nz, ny, nx = m.shape
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                if not m[z, y, x]:
                    continue
                x1 = x
                while x1 + 1 < nx and m[z, y, x1 + 1] and x1 + 1 - x < max_side_blocks:
                    x1 += 1
                y1 = y
                while (y1 + 1 < ny and y1 + 1 - y < max_side_blocks
                       and m[z, y1 + 1, x:x1 + 1].all()):
                    y1 += 1
                z1 = z
                while (dim == 3 and z1 + 1 < nz and z1 + 1 - z < max_side_blocks
                       and m[z1 + 1, y:y1 + 1, x:x1 + 1].all()):
                    z1 += 1
                m[z:z1 + 1, y:y1 + 1, x:x1 + 1] = False
                lo = [x * block, y * block, z * block if dim == 3 else 0]
                hi = [(x1 + 1) * block - 1, (y1 + 1) * block - 1,
                      (z1 + 1) * block - 1 if dim == 3 else 0]
                boxes.append(lo + hi)
    return np.asarray(boxes, dtype=np.int32).reshape(-1, 6)


def _chop_uniform(n, side, dim):
    boxes = []
    nz = n[2] if dim == 3 else 1
    for z0 in range(0, nz, side):
        for y0 in range(0, n[1], side):
            for x0 in range(0, n[0], side):
                lo = [x0, y0, z0 if dim == 3 else 0]
                hi = [min(x0 + side, n[0]) - 1, min(y0 + side, n[1]) - 1,
                      (min(z0 + side, nz) - 1) if dim == 3 else 0]
                boxes.append(lo + hi)
    return np.asarray(boxes, dtype=np.int32)


def _nested_block_mask(rng, dim, n_cells, block, centers, nbox, side_lo, side_hi,
                       parent_ok=None):
    """Mark blocks touched by random boxes (sides U{side_lo..side_hi} cells)
    centred near the given points; optionally restricted by parent_ok."""
    nb = [n_cells[a] // block if a < dim else 1 for a in range(3)]
    mask = np.zeros((nb[2], nb[1], nb[0]), dtype=bool)
    for c in centers:
        for _ in range(nbox):
            side = rng.integers(side_lo, side_hi + 1, size=3)
            jitter = rng.normal(0.0, 0.04, size=3)
            lo = []
            hi = []
            for a in range(3):
                if a >= dim:
                    lo.append(0)
                    hi.append(0)
                    continue
                ctr = (c[a] + jitter[a]) * n_cells[a]
                l = int(math.floor(ctr - side[a] / 2))
                h = l + int(side[a]) - 1
                l = max(l, 0)
                h = min(h, n_cells[a] - 1)
                lo.append(l // block)
                hi.append(h // block)
            if dim == 2:
                mask[0, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = True
            else:
                mask[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = True
    if parent_ok is not None:
        mask &= parent_ok
    return mask


def _parent_ok_mask(parent_mask, parent_block, child_block, ratio, dim):
    """Child blocks whose footprint grown by one parent cell (in every
    direction, diagonals included) lies inside the parent mask; beyond the
    physical boundary no buffer is needed (proper nesting)."""
    cells = parent_mask
    for ax in ([0, 1, 2] if dim == 3 else [1, 2]):
        cells = np.repeat(cells, parent_block, axis=ax)
    pad = [(1, 1)] * 3 if dim == 3 else [(0, 0), (1, 1), (1, 1)]
    padded = np.pad(cells, pad, mode="constant", constant_values=True)
    er = np.ones_like(cells)
    offs = [-1, 0, 1]
    for dz in (offs if dim == 3 else [0]):
        for dy in offs:
            for dx in offs:
                z0 = 1 + dz if dim == 3 else 0
                sl = padded[z0:z0 + cells.shape[0], 1 + dy:1 + dy + cells.shape[1],
                            1 + dx:1 + dx + cells.shape[2]]
                er &= sl
    cb = child_block // ratio
    if dim == 3:
        nzc, nyc, nxc = (s // cb for s in er.shape)
        v = er[:nzc * cb, :nyc * cb, :nxc * cb].reshape(nzc, cb, nyc, cb, nxc, cb)
        return v.all(axis=(1, 3, 5))
    nyc, nxc = er.shape[1] // cb, er.shape[2] // cb
    v = er[:, :nyc * cb, :nxc * cb].reshape(1, nyc, cb, nxc, cb)
    return v.all(axis=(2, 4))


# ---------------------------------------------------------------------------
# configurations
# ---------------------------------------------------------------------------

def config1() -> Problem:
    """2-D sine problem: coarse 64x64, fine box (32,32)-(95,95) at ratio 2."""
    lev0 = Level((1, 1, 1), np.array([[0, 0, 0, 63, 63, 0]], dtype=np.int32))
    lev1 = Level((2, 2, 1), np.array([[32, 32, 0, 95, 95, 0]], dtype=np.int32))
    p = Problem(dim=2, n0=(64, 64, 1), xlo=(0.0, 0.0, 0.0), xup=(1.0, 1.0, 1.0),
                levels=[lev0, lev1], name="config1_2d_sine")
    # -lap(u) = 2 pi^2 sin(pi x) sin(pi y); SAMRAI solves div(grad u) = rhs,
    # so the rhs passed is -f (FAC_staticrefinement/fortran/facpoisson2d.m4).
    def rhs(X, Y, Z):
        return -2.0 * math.pi ** 2 * np.sin(math.pi * X) * np.sin(math.pi * Y)
    _finish(p, rhs)
    return p


def exact_config1(X, Y):
    return np.sin(math.pi * X) * np.sin(math.pi * Y)


def _finish(p: Problem, rhs, dfn=None, cfn=None):
    p.f = [fill_cell_field(p, ln, 0, rhs) for ln in range(p.nlev)]
    p.u0 = [np.zeros(field_size(p, ln, 1)) for ln in range(p.nlev)]
    if dfn is not None:
        p.d_variable = True
        p.d = [fill_side_field(p, ln, dfn) for ln in range(p.nlev)]
    if cfn is not None:
        p.c_kind = 2
        p.c = [fill_cell_field(p, ln, 0, cfn) for ln in range(p.nlev)]


def gaussian_bumps(seed, dim, nbump=4, width=0.05):
    rng = np.random.default_rng(seed)
    centers = rng.uniform(0.25, 0.75, size=(nbump, 3))
    if dim == 2:
        centers[:, 2] = 0.0
    amps = rng.normal(0.0, 1.0, size=nbump)
    return centers, amps, width


def _bump_rhs(centers, amps, width, dim):
    def rhs(X, Y, Z):
        out = np.zeros_like(X)
        for c, a in zip(centers, amps):
            r2 = (X - c[0]) ** 2 + (Y - c[1]) ** 2
            if dim == 3:
                r2 = r2 + (Z - c[2]) ** 2
            out += a * np.exp(-r2 / (2.0 * width ** 2))
        return out
    return rhs


class _FourierField:
    """Smooth Gaussian random field: sum of random Fourier modes, evaluable
    at points or (fast, through a GEMM) on tensor-product grids."""

    def __init__(self, k, phase, amp, scale, post=None):
        self.k, self.phase, self.amp, self.scale = k, phase, amp, scale
        self.post = post

    def __call__(self, X, Y, Z):
        out = np.zeros_like(X)
        for m in range(len(self.amp)):
            out += self.amp[m] * np.cos(self.k[m, 0] * X + self.k[m, 1] * Y +
                                        self.k[m, 2] * Z + self.phase[m])
        out *= self.scale
        return self.post(out) if self.post else out

    def grid(self, xs, ys, zs):
        c = self.amp * np.exp(1j * self.phase)
        ex = np.exp(1j * np.outer(self.k[:, 0], xs))          # (M, nx)
        ey = np.exp(1j * np.outer(self.k[:, 1], ys))          # (M, ny)
        ez = np.exp(1j * np.outer(self.k[:, 2], zs))          # (M, nz)
        t = (ez.T[:, None, :] * ey.T[None, :, :]) * c        # (nz, ny, M)
        g = (t.reshape(-1, len(c)) @ ex).real.reshape(len(zs), len(ys), len(xs))
        g *= self.scale
        return self.post(g) if self.post else g

    def exp(self):
        return _FourierField(self.k, self.phase, self.amp, self.scale, post=np.exp)


def random_field(seed, dim, corr_len=0.1, contrast=1e3, nmodes=64):
    """Smooth Gaussian random field g (random Fourier features with a
    Gaussian spectrum of correlation length corr_len), scaled so that
    exp(g) spans about ``contrast``."""
    rng = np.random.default_rng(seed + 1000)
    k = rng.normal(0.0, 1.0 / corr_len, size=(nmodes, 3))
    if dim == 2:
        k[:, 2] = 0.0
    phase = rng.uniform(0.0, 2 * math.pi, size=nmodes)
    amp = rng.normal(0.0, 1.0, size=nmodes) * math.sqrt(2.0 / nmodes)
    raw = _FourierField(k, phase, amp, 1.0)
    g = np.linspace(0.0, 1.0, 33)
    s = raw.grid(g, g, g if dim == 3 else np.zeros(1))
    scale = math.log(contrast) / max(float(s.max() - s.min()), 1e-12)
    return _FourierField(k, phase, amp, scale)


def build_3d_hierarchy(seed, n0, max_patch=32, nbox=(6, 6), side=(8, 48),
                       nlev=3, block=8, max_patch0=None):
    """Coarse n0^3 chopped into max_patch^3 patches; finer levels (ratio 2)
    are unions of seeded random boxes (sides U{side}) around 4 seeded
    Gaussian centres, clipped for proper nesting and chopped to max_patch."""
    dim = 3
    centers, amps, width = gaussian_bumps(seed, dim)
    rng = np.random.default_rng(seed)
    levels = [Level((1, 1, 1), _chop_uniform([n0, n0, n0], max_patch0 or max_patch, dim))]
    parent_mask = np.ones((n0 // block, n0 // block, n0 // block), dtype=bool)
    n_cells = n0
    for ln in range(1, nlev):
        n_cells *= 2
        ok = _parent_ok_mask(parent_mask, block, block, 2, dim)
        mask = _nested_block_mask(rng, dim, [n_cells] * 3, block, centers,
                                  nbox[ln - 1], side[0], side[1], parent_ok=ok)
        boxes = _mask_to_boxes(mask, block, max_patch // block, dim)
        levels.append(Level((2, 2, 2), boxes))
        parent_mask = mask
    return levels, (centers, amps, width)


def config2(seed=2, n0=128) -> Problem:
    """3-D batched uneven patches: coarse 128^3 in 32^3 patches, levels 1-2
    of seeded random boxes around 4 Gaussian bumps, f = sum of the bumps."""
    levels, (centers, amps, width) = build_3d_hierarchy(seed, n0)
    p = Problem(dim=3, n0=(n0, n0, n0), xlo=(0.0, 0.0, 0.0), xup=(1.0, 1.0, 1.0),
                levels=levels, name="config2_3d_bumps")
    _finish(p, _bump_rhs(centers, amps, width, 3))
    return p


def config3(seed=3) -> Problem:
    """Config-1 hierarchy with D = exp(g), g a Gaussian random field with
    correlation length 0.1 and 1e3 contrast; C = 0."""
    p = config1()
    p.name = "config3_2d_varcoef"
    d = random_field(seed, 2).exp()
    p.d_variable = True
    p.d = [fill_side_field(p, ln, d) for ln in range(p.nlev)]
    return p


def config5_problem(seed, n0=None, nbox=(3, 3)) -> Problem:
    """One of the 64 batched 3-D variable-coefficient problems: coarse
    n0^3 (n0 ~ U{64..128}, a multiple of 8) in patches of at most 32^3,
    levels 1-2 (ratio 2) in patches of 8..16 cells per side, D = exp(g)."""
    rng = np.random.default_rng(10_000 + seed)
    if n0 is None:
        n0 = int(rng.integers(8, 17)) * 8
    levels, (centers, amps, width) = build_3d_hierarchy(seed, n0, nbox=nbox, max_patch=16,
                                                        max_patch0=32)
    p = Problem(dim=3, n0=(n0, n0, n0), xlo=(0.0, 0.0, 0.0), xup=(1.0, 1.0, 1.0),
                levels=levels, name=f"config5_problem{seed}")
    _finish(p, _bump_rhs(centers, amps, width, 3), dfn=random_field(seed, 3).exp())
    return p


def small_3d(seed=7, n0=32) -> Problem:
    """A small 3-D three-level problem for quick parity tests."""
    levels, (centers, amps, width) = build_3d_hierarchy(
        seed, n0, max_patch=16, nbox=(3, 3), side=(8, 24), block=4)
    p = Problem(dim=3, n0=(n0, n0, n0), xlo=(0.0, 0.0, 0.0), xup=(1.0, 1.0, 1.0),
                levels=levels, name="small_3d")
    _finish(p, _bump_rhs(centers, amps, 0.1, 3))
    return p


def config5_cost(seed) -> int:
    """Coarse cells of config-5 problem `seed` (its n0 draw, without building
    the problem): the weight of the problem when problems are spread over
    ranks."""
    n0 = int(np.random.default_rng(10_000 + seed).integers(8, 17)) * 8
    return n0 ** 3


def config5(nprob=64, first_seed=0, workers=None, seeds=None):
    """64 independent 3-D variable-coefficient problems (seeds 0..63, or the
    given seeds), generated in parallel worker processes."""
    if seeds is None:
        seeds = list(range(first_seed, first_seed + nprob))
    seeds = list(seeds)
    if workers is None:
        import os
        workers = min(len(seeds), os.cpu_count() or 1, 32)
    if workers <= 1:
        return [config5_problem(s) for s in seeds]
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_config5_worker, seeds)


def _config5_worker(seed):
    try:
        from threadpoolctl import threadpool_limits
        with threadpool_limits(1):
            return config5_problem(seed)
    except ImportError:
        return config5_problem(seed)


# ---------------------------------------------------------------------------
# virtual coarse levels (multigrid coarsest-level solve for the fast variant)
# ---------------------------------------------------------------------------

def extend_hierarchy(prob: Problem, min_cells: int = 8, k: Optional[int] = None) -> Problem:
    """Prepend k levels that coarsen the domain by 2 (default: until the
    coarsest has fewer than 2*min_cells cells per side or an odd count).

    The added levels each cover the whole domain, so every one of their
    cells is covered by the next finer level: the composite problem, its
    weights and its residual norm are unchanged, and the FAC cycle becomes
    a full multigrid V-cycle whose coarsest solve is cheap (SAMRAI reaches
    the same effect with its hypre coarse solver, CellPoissonFACOps.C:
    1741-1781).  D on an added level is the mean of the finer faces on each
    coarse face; f and u0 there are zero (fully covered cells)."""
    dim = prob.dim
    n = list(prob.n0[:dim])
    if k is None:
        k = 0
        while all(x % 2 == 0 and x // 2 >= min_cells for x in n):
            n = [x // 2 for x in n]
            k += 1
    else:
        assert all(x % (2 ** k) == 0 for x in n), "domain not divisible by 2^k"
    if k == 0:
        return prob
    # level 0 of the input must cover the domain
    b0 = prob.levels[0].boxes
    cov = int(np.prod(b0[:, 3:] - b0[:, :3] + 1, axis=1).sum())
    assert cov == int(np.prod([prob.n0[a] for a in range(dim)])), "level 0 must cover the domain"
    levels = []
    for j in range(k, 0, -1):
        m = [x // (2 ** j) for x in prob.n0[:dim]]
        hi = [m[a] - 1 if a < dim else 0 for a in range(3)]
        ratio = (1, 1, 1) if j == k else tuple(2 if a < dim else 1 for a in range(3))
        levels.append(Level(ratio, np.array([[0, 0, 0] + hi], dtype=np.int32)))
    first_orig = Level(tuple(2 if a < dim else 1 for a in range(3)), prob.levels[0].boxes)
    levels.append(first_orig)
    levels.extend(prob.levels[1:])
    n0 = tuple(prob.n0[a] // (2 ** k) if a < dim else 1 for a in range(3))
    ext = Problem(dim=dim, n0=n0, xlo=prob.xlo, xup=prob.xup, levels=levels,
                  d_variable=prob.d_variable, d_const=prob.d_const, c_kind=prob.c_kind,
                  c_const=prob.c_const, name=prob.name + f"+{k}mg")
    ext.virtual_levels = k
    ext.f = [np.zeros(field_size(ext, ln, 0)) for ln in range(k)] + list(prob.f)
    ext.u0 = [np.zeros(field_size(ext, ln, 1)) for ln in range(k)] + list(prob.u0)
    if prob.c_kind == 2:
        ext.c = [np.zeros(field_size(ext, ln, 0)) for ln in range(k)] + list(prob.c)
    if prob.d_variable:
        dk = [None] * k + list(prob.d)
        # dense side grids of the original level 0 (covers the domain)
        dense = _dense_side(prob, 0, prob.d[0])
        for ln in range(k - 1, -1, -1):
            dense = [_coarsen_dense_side(dense[a], a, dim) for a in range(dim)]
            dk[ln] = np.concatenate([dense[a].reshape(-1) for a in range(dim)])
        ext.d = dk
    return ext


def _dense_side(prob: Problem, ln: int, d: np.ndarray):
    """Per-axis dense side arrays (z, y, x) over the domain of level ln from
    the patch side data of a level that covers the domain."""
    dim = prob.dim
    lo, hi = prob.domain(ln)
    n = [hi[a] - lo[a] + 1 for a in range(3)]
    out = []
    for a in range(dim):
        e = list(n)
        e[a] += 1
        out.append(np.zeros((e[2], e[1], e[0])))
    off = 0
    for b in prob.levels[ln].boxes:
        for a in range(dim):
            lo_b = b[:3].copy()
            hi_b = b[3:].copy()
            hi_b[a] += 1
            ext = hi_b - lo_b + 1
            cnt = int(np.prod(ext))
            v = d[off:off + cnt].reshape(ext[2], ext[1], ext[0])
            out[a][lo_b[2]:hi_b[2] + 1, lo_b[1]:hi_b[1] + 1, lo_b[0]:hi_b[0] + 1] = v
            off += cnt
    return out


def _coarsen_dense_side(s: np.ndarray, a: int, dim: int):
    """Mean of the 2^(dim-1) fine faces on each coarse face of axis a."""
    ax = {0: 2, 1: 1, 2: 0}[a]          # numpy axis of index a
    # keep every other face along the normal axis
    sl = [slice(None)] * 3
    sl[ax] = slice(0, None, 2)
    t = s[tuple(sl)]
    tang = [x for x in (0, 1, 2) if x != a and x < dim]
    for tt in tang:
        nax = {0: 2, 1: 1, 2: 0}[tt]
        t = 0.5 * (np.take(t, range(0, t.shape[nax], 2), axis=nax) +
                   np.take(t, range(1, t.shape[nax], 2), axis=nax))
    return np.ascontiguousarray(t)
