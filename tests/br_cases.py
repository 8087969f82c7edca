"""Cases of the regrid step (tagging + Berger-Rigoutsos) shared by the
fixture generator (tests/golden/make_br_fixtures.py) and the tests.

The tagged field is a sum of bumps a (r^2 - |x - c|^2)^2 (zero outside
radius r) with dyadic centres, radii and amplitudes on a grid of spacing
2^-k, so every value is a short chain of IEEE additions and products of
exactly representable numbers: the same bits on every machine.
"""
import numpy as np

from samrai_b200 import configs

# name: dim, domain cells, patch side, bumps (centre, r, amplitude),
# threshold, bound boxes (None: the domain), min_box, max_box (0: none),
# efficiency tolerance, combine efficiency
CASES = {
    "br_2d": dict(dim=2, n=128, side=64,
                  bumps=[((0.25, 0.375), 0.125, 64.0), ((0.71875, 0.65625), 0.0625, 512.0),
                         ((0.5, 0.875), 0.09375, 128.0)],
                  threshold=1.0 / 16384, bound=None, min_box=(4, 4), max_box=(0, 0),
                  efficiency=0.8, combine=0.8),
    "br_2d_small_boxes": dict(dim=2, n=96, side=32,
                              bumps=[((0.3125, 0.3125), 0.1875, 32.0),
                                     ((0.6875, 0.75), 0.125, 96.0)],
                              threshold=1.0 / 2048, bound=[[0, 0, 0, 47, 95, 0],
                                                           [48, 0, 0, 95, 95, 0]],
                              min_box=(2, 2), max_box=(24, 24), efficiency=0.7, combine=0.85),
    "br_3d": dict(dim=3, n=48, side=24,
                  bumps=[((0.25, 0.3125, 0.375), 0.1875, 16.0),
                         ((0.6875, 0.625, 0.5625), 0.125, 64.0)],
                  threshold=1.0 / 4096, bound=None, min_box=(2, 2, 2), max_box=(0, 0, 0),
                  efficiency=0.85, combine=0.8),
    "br_3d_eff": dict(dim=3, n=32, side=16,
                      bumps=[((0.375, 0.5, 0.4375), 0.25, 8.0),
                             ((0.75, 0.25, 0.75), 0.125, 32.0)],
                      threshold=1.0 / 8192, bound=None, min_box=(2, 2, 2),
                      max_box=(12, 12, 12), efficiency=0.9, combine=0.75),
}


def problem(name):
    """One-level configs.Problem over the case's domain (the tag level) with
    u set on every ghost-1 patch array."""
    c = CASES[name]
    dim, n, side = c["dim"], c["n"], c["side"]
    n0 = tuple([n] * dim + [1] * (3 - dim))
    boxes = configs._chop_uniform(list(n0), side, dim)
    p = configs.Problem(dim=dim, n0=n0, xlo=(0.0,) * 3, xup=(1.0,) * 3,
                        levels=[configs.Level((1, 1, 1), boxes)], name=name)
    h = 1.0 / n
    u = []
    for b in boxes:
        lo, hi = b[:3], b[3:]
        axes = []
        for a in range(3):
            if a < dim:
                axes.append((np.arange(lo[a] - 1, hi[a] + 2) + 0.5) * h)
            else:
                axes.append(np.array([0.0]))
        z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
        v = np.zeros(x.shape)
        for cen, r, amp in c["bumps"]:
            q = r * r - (x - cen[0]) ** 2 - (y - cen[1]) ** 2
            if dim == 3:
                q = q - (z - cen[2]) ** 2
            q = np.maximum(q, 0.0)
            v = v + amp * (q * q)
        u.append(v.reshape(-1))
    p.u0 = [np.concatenate(u)]
    p.f = [np.zeros(configs.field_size(p, 0, 0))]
    return p


def bound_boxes(name):
    c = CASES[name]
    if c["bound"] is not None:
        return np.array(c["bound"], dtype=np.int32)
    n, dim = c["n"], c["dim"]
    hi = [n - 1 if a < dim else 0 for a in range(3)]
    return np.array([[0, 0, 0] + hi], dtype=np.int32)


def patch_arrays(p, arr, g):
    """Per-patch pieces of a level array (ghost width g)."""
    out, off = [], 0
    for b in p.levels[0].boxes:
        cnt = int(np.prod([b[3 + a] - b[a] + 1 + (2 * g if a < p.dim else 0) for a in range(3)]))
        out.append(arr[off:off + cnt])
        off += cnt
    return out


def sorted_boxes(boxes):
    b = np.asarray(boxes, dtype=np.int64).reshape(-1, 6)
    return b[np.lexsort(b.T[::-1])]
