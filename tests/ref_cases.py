"""Problems whose full FAC solves by the reference's own solver
(oracle/_ref/fac_ref_driver: SAMRAI's CellPoissonFACSolver, its schedules,
coarse-fine boundaries, norms and FAC loop, with its Fortran kernels
translated to C) are stored as golden fixtures in tests/golden/ref_*.npz.

Each case: (problem builder, solver parameters, Robin coefficients -- a
constant triple per side, "faces" for robin_face_coefs, or None for
Dirichlet u = 0 -- and whether the fixture keeps the full solution arrays).
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


def robin_face_coefs(prob, ln, loc):
    """Robin (a, b, g) varying along every side of the domain, the same
    polynomial of the face-centre coordinates that fac_ref_driver's
    position-dependent coefficient object evaluates: t = sum over the
    tangential axes of x = xlo + (i + 0.5) dx (level ln's dx), a = 1 +
    t/4, b = 1/2 + t/8, g = t/10 - 1/20 + loc/100.  Returns the (n, 3)
    array over the level's domain face, lowest tangential axis fastest."""
    dim = prob.dim
    a_n = loc // 2
    lo, hi = prob.domain(ln)
    dx = prob.dx(ln)
    tang = [t for t in range(dim) if t != a_n]
    axes = [np.arange(lo[t], hi[t] + 1) for t in tang]
    grids = np.meshgrid(*axes[::-1], indexing="ij")[::-1]
    t = np.zeros(grids[0].shape)
    for g, ax in zip(grids, tang):
        t = t + (prob.xlo[ax] + (g.astype(np.float64) + 0.5) * dx[ax])
    t = t.reshape(-1)
    return np.stack([1.0 + 0.25 * t, 0.5 + 0.125 * t, 0.1 * t - 0.05 + 0.01 * loc], axis=1)


def all_face_coefs(prob):
    return {(ln, loc): robin_face_coefs(prob, ln, loc)
            for ln in range(prob.nlev) for loc in range(2 * prob.dim)}


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
    # Robin coefficients varying along the boundary (robin_face_coefs)
    "robin_faces_2d": (configs.config1, TIGHT, "faces", True),
    "robin_faces_3d": (configs.small_3d, dict(BASE, coarse_tol=1e-300, coarse_max_it=100),
                       "faces", False),
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
