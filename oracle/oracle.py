"""ctypes binding of the CPU oracle (fac_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Imported by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the
samrai_b200 package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libfacoracle.so")
_lib = None

U, F, E, R, TR, W, C = range(7)
SD, SFLUX = range(2)
CELL_GHOST = [1, 0, 1, 0, 0, 0, 0]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def build_timing():
    """Compile the -O3 -march=native timing build of the oracle into a fresh
    temporary directory (the CPU it targets is the one running this) and
    return its path; the results are bit-identical to the default build."""
    import tempfile
    d = tempfile.mkdtemp(prefix="facoracle_timing_")
    subprocess.run(["make", "-s", "-C", _HERE, "timing", f"TIMING_DIR={d}"], check=True)
    return os.path.join(d, "libfacoracle.so")


def use_library(path):
    """Load the oracle from `path` (a timing build) instead of the default
    build; must precede the first call into the oracle in this process."""
    global _LIB_PATH
    if _lib is not None and path != _LIB_PATH:
        raise RuntimeError("oracle library already loaded")
    _LIB_PATH = path


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, ip, dp, dp, ctypes.c_int, ip, ip, ip]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_set_poisson.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_double]
        L.orc_set_bc.argtypes = [ctypes.c_void_p, dp, dp, dp]
        L.orc_set_bc_faces.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp]
        L.orc_set_params.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_int, ctypes.c_int]
        for n in ("orc_field_size", "orc_side_size"):
            getattr(L, n).restype = ctypes.c_long
            getattr(L, n).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_oside_size.restype = ctypes.c_long
        L.orc_oside_size.argtypes = [ctypes.c_void_p, ctypes.c_int]
        for n in ("orc_get_field", "orc_set_field", "orc_get_side", "orc_set_side"):
            getattr(L, n).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp]
        L.orc_get_oside.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.orc_ghost_fill.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 4
        L.orc_smooth.restype = ctypes.c_int
        L.orc_smooth.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_double, dp]
        L.orc_comp_residual.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 5
        L.orc_restrict.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 3
        L.orc_restrict_solution.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 2
        L.orc_prolong_correct.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 3
        L.orc_compute_weights.argtypes = [ctypes.c_void_p]
        L.orc_rms_norm.restype = ctypes.c_double
        L.orc_rms_norm.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_solve_coarsest.restype = ctypes.c_int
        L.orc_solve_coarsest.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 3
        L.orc_fac_cycle.argtypes = [ctypes.c_void_p]
        L.orc_solve.restype = ctypes.c_int
        L.orc_solve.argtypes = [ctypes.c_void_p, ip, dp, dp]
        L.orc_coarse_sweeps.restype = ctypes.c_long
        L.orc_coarse_sweeps.argtypes = [ctypes.c_void_p]
        L.orc_reset_stats.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Oracle:
    """One FAC hierarchy on the CPU, set up like CellPoissonFACSolver."""

    def __init__(self, prob, params=None, bc=None, bc_faces=None):
        L = lib()
        self.prob = prob
        dim = prob.dim
        n0 = np.array(prob.n0, dtype=np.int32)
        xlo = np.array(prob.xlo, dtype=np.float64)
        xup = np.array(prob.xup, dtype=np.float64)
        ratio = np.array([lv.ratio for lv in prob.levels], dtype=np.int32).reshape(-1)
        npatch = np.array([len(lv.boxes) for lv in prob.levels], dtype=np.int32)
        boxes = np.concatenate([lv.boxes for lv in prob.levels]).astype(np.int32).reshape(-1)
        self._keep = (n0, xlo, xup, ratio, npatch, boxes)
        self.h = L.orc_create(dim, _ip(n0), _dp(xlo), _dp(xup), prob.nlev, _ip(ratio),
                              _ip(npatch), _ip(boxes))
        if not self.h:
            raise RuntimeError("orc_create failed")
        L.orc_set_poisson(self.h, int(prob.d_variable), float(prob.d_const),
                          int(prob.c_kind), float(prob.c_const))
        if bc is not None:
            a, b, g = (np.asarray(x, dtype=np.float64) for x in bc)
            L.orc_set_bc(self.h, _dp(a), _dp(b), _dp(g))
        # per-face Robin coefficients: {(level, location): (n, 3) array}
        self._faces = {}
        for (ln, loc), abg in (bc_faces or {}).items():
            arr = np.ascontiguousarray(abg, dtype=np.float64).reshape(-1)
            self._faces[ln, loc] = arr
            L.orc_set_bc_faces(self.h, int(ln), int(loc), _dp(arr))
        p = dict(max_cycles=100, residual_tol=1e-300, relative_residual_tol=1e-10,
                 pre_sweeps=2, post_sweeps=2, coarse_tol=1e-8, coarse_max_it=500, ewing=1)
        if params:
            p.update(params)
        self.params = p
        L.orc_set_params(self.h, p["max_cycles"], p["residual_tol"], p["relative_residual_tol"],
                         p["pre_sweeps"], p["post_sweeps"], p["coarse_tol"],
                         p["coarse_max_it"], p["ewing"])
        for ln in range(prob.nlev):
            if prob.f:
                self.set(F, ln, prob.f[ln])
            if prob.u0:
                self.set(U, ln, prob.u0[ln])
            if prob.d_variable:
                self.set_side(SD, ln, prob.d[ln])
            if prob.c_kind == 2:
                self.set(C, ln, prob.c[ln])

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def size(self, fid, ln):
        return lib().orc_field_size(self.h, fid, ln)

    def get(self, fid, ln):
        out = np.empty(self.size(fid, ln))
        lib().orc_get_field(self.h, fid, ln, _dp(out))
        return out

    def set(self, fid, ln, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        assert arr.size == self.size(fid, ln), (arr.size, self.size(fid, ln))
        lib().orc_set_field(self.h, fid, ln, _dp(arr))

    def get_side(self, sid, ln):
        out = np.empty(lib().orc_side_size(self.h, sid, ln))
        lib().orc_get_side(self.h, sid, ln, _dp(out))
        return out

    def set_side(self, sid, ln, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        lib().orc_set_side(self.h, sid, ln, _dp(arr))

    def get_oside(self, ln):
        out = np.empty(lib().orc_oside_size(self.h, ln))
        lib().orc_get_oside(self.h, ln, _dp(out))
        return out

    # operations -----------------------------------------------------------
    def ghost_fill(self, fid, ln, with_coarse, homogeneous):
        lib().orc_ghost_fill(self.h, fid, ln, int(with_coarse), int(homogeneous))

    def smooth(self, fid_e, fid_r, ln, nsweeps, tol=-1.0):
        mr = ctypes.c_double(0.0)
        n = lib().orc_smooth(self.h, fid_e, fid_r, ln, nsweeps, tol, ctypes.byref(mr))
        return n, mr.value

    def comp_residual(self, fid_r, fid_u, fid_f, ln, error_eq):
        lib().orc_comp_residual(self.h, fid_r, fid_u, fid_f, ln, int(error_eq))

    def restrict(self, fid_src, fid_dst, dest_ln):
        lib().orc_restrict(self.h, fid_src, fid_dst, dest_ln)

    def restrict_solution(self, fid, dest_ln):
        lib().orc_restrict_solution(self.h, fid, dest_ln)

    def prolong_correct(self, fid_src, fid_dst, dest_ln):
        lib().orc_prolong_correct(self.h, fid_src, fid_dst, dest_ln)

    def compute_weights(self):
        lib().orc_compute_weights(self.h)

    def rms_norm(self, fid):
        return lib().orc_rms_norm(self.h, fid)

    def solve_coarsest(self):
        return lib().orc_solve_coarsest(self.h, E, R, 0)

    def fac_cycle(self):
        lib().orc_fac_cycle(self.h)

    def coarse_sweeps(self):
        return lib().orc_coarse_sweeps(self.h)

    def solve(self):
        it = ctypes.c_int(0)
        res = ctypes.c_double(0.0)
        hist = np.zeros(self.params["max_cycles"] + 1)
        ok = lib().orc_solve(self.h, ctypes.byref(it), ctypes.byref(res), _dp(hist))
        return bool(ok), it.value, res.value, hist[:it.value + 1]
