"""Problems whose full FAC solves by the reference's own solver
(oracle/_ref/fac_ref_driver: SAMRAI's CellPoissonFACSolver, its schedules,
coarse-fine boundaries, norms and FAC loop, with its Fortran kernels
translated to C) are stored as golden fixtures in tests/golden/ref_*.npz.

Each case: (problem builder, solver parameters, Robin coefficients or None
for Dirichlet u = 0, whether the fixture keeps the full solution arrays).
Every fixture keeps, per level, SHA-256 digests of the solution's bytes
(interior cells, and all cells with the ghost cells), a fingerprint and
every SAMPLE-th value; the small 2-D cases keep the full arrays as well.
"""
import hashlib
import math

import numpy as np

from samrai_b200 import configs

# FACPreconditioner / CellPoissonFACOps inputs: the reference's defaults for
# the coarsest solve (red-black, tolerance 1e-8, at most 500 sweeps) unless
# a case says otherwise
BASE = dict(max_cycles=100, residual_tol=1e-300, relative_residual_tol=1e-10, pre_sweeps=2,
            post_sweeps=2, coarse_tol=1e-8, coarse_max_it=500, ewing=1)


def mixed_parity_2d():
    """Config 1 with its coarse level cut into six patches whose first cells
    lie on both parities of i + j, so the patch-relative red-black colouring
    (solv_cellpoissonfacops2d.f:140-147) differs between neighbours."""
    p = configs.config1()
    xs = [(0, 20), (21, 42), (43, 63)]
    ys = [(0, 30), (31, 63)]
    boxes = [[x0, y0, 0, x1, y1, 0] for (y0, y1) in ys for (x0, x1) in xs]
    p.levels[0] = configs.Level((1, 1, 1), np.asarray(boxes, dtype=np.int32))
    p.name = "mixed_parity_2d"

    def rhs(X, Y, Z):
        return -2.0 * math.pi ** 2 * np.sin(math.pi * X) * np.sin(math.pi * Y)
    configs._finish(p, rhs)
    return p


def c_field_2d():
    """Config 3 (variable D) with a variable C field, C = -5 (1 + x + y)."""
    p = configs.config3()
    p.name = "c_field_2d"
    p.c_kind = 2
    p.c = [configs.fill_cell_field(p, ln, 0, lambda X, Y, Z: -5.0 * (1.0 + X + Y))
           for ln in range(p.nlev)]
    return p


def small_3d_varcoef():
    p = configs.small_3d(seed=7)
    p.name = "small_3d_varcoef"
    d = configs.random_field(11, 3).exp()
    p.d_variable = True
    p.d = [configs.fill_side_field(p, ln, d) for ln in range(p.nlev)]
    return p


def config2_mg():
    return configs.extend_hierarchy(configs.config2(), k=4)


# Robin a u + b du/dn = g on the four sides (location index 0..3)
ROBIN = (np.array([1.0, 2.0, 1.0, 0.5, 0, 0]), np.array([0.5, 1.0, 0.25, 1.0, 0, 0]),
         np.array([0.1, -0.2, 0.05, 0.3, 0, 0]))

# the coarsest solve run to its sweep limit on every cycle (tolerance 1e-300):
# with the reference's default 1e-8 the 2-D cases stall just above the
# 1e-10 relative target and stop at max_cycles
TIGHT = dict(BASE, coarse_tol=1e-300)

CASES = {
    "config1": (configs.config1, BASE, None, True),
    "config1_tight": (configs.config1, TIGHT, None, True),
    "config3": (configs.config3, BASE, None, True),
    "config3_tight": (configs.config3, TIGHT, None, True),
    "mixed_parity_2d": (mixed_parity_2d, dict(BASE, coarse_tol=1e-300, coarse_max_it=200),
                        None, True),
    "robin_2d": (configs.config1, TIGHT, ROBIN, True),
    "c_field_2d": (c_field_2d, TIGHT, None, True),
    "small_3d": (configs.small_3d, dict(BASE, coarse_tol=1e-300, coarse_max_it=100), None,
                 False),
    "small_3d_varcoef": (small_3d_varcoef, dict(BASE, coarse_tol=1e-300, coarse_max_it=100),
                         None, False),
    "config2_mg": (config2_mg, dict(BASE, coarse_tol=1e-300, coarse_max_it=20), None, False),
}

# every SAMPLE-th element of each level's solution, kept for cases whose
# full arrays would be too large for a fixture
SAMPLE = 97


def summarize(u):
    """Size-independent fingerprint of one level's solution array."""
    return np.array([u.size, u.sum(), (u * u).sum(), np.abs(u).max()])


def interior_mask(prob, ln):
    """Interior cells of a level's ghost-1 canonical cell array."""
    n = configs.field_size(prob, ln, 1)
    m = np.zeros(n, dtype=bool)
    idx = np.arange(n)
    for _, _, v in configs.patch_views(prob, ln, idx, 1):
        inner = v[1:-1, 1:-1, 1:-1] if prob.dim == 3 else v[:, 1:-1, 1:-1]
        m[inner.reshape(-1)] = True
    return m


def digest(a):
    """SHA-256 of the little-endian float64 bytes of an array (as uint8)."""
    h = hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).digest()
    return np.frombuffer(h, dtype=np.uint8).copy()
