"""Python binding of the B200 FAC library (C ABI in include/samrai_fac_b200.h).

Two layers, mirroring the reference's own split:

* :class:`FacContext` -- one-to-one with the C ABI: a batch of problems on
  one GPU and the FACOperatorStrategy level operators
  (solv/FACOperatorStrategy.h:83-364) plus the whole solve.
* :class:`CellPoissonFACSolver` -- the drop-in for solv::CellPoissonFACSolver
  (solv/CellPoissonFACSolver.h:116-475): same method names, input keys and
  defaults, driving a FacContext.

There is no CPU fallback: the CUDA library must be built
(``python -m samrai_b200.build``) and a GPU present, or the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from typing import List, Optional, Sequence

import numpy as np

from . import build as _build

U, F, E, R, TR, W, C = range(7)
CELL_GHOST = [1, 0, 1, 0, 0, 0, 0]

_lib = None


class FacError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"FAC error {code}: {msg}")
        self.code = code


def library_path():
    return _build.LIB


def load_library(build_if_missing=True):
    """Load libsamrai_fac_b200.so (building it in-tree if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise FileNotFoundError(f"{path} is missing; run python -m samrai_b200.build")
        _build.build()
    L = ctypes.CDLL(path)
    vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    szp = ctypes.POINTER(ctypes.c_size_t)
    fp = ctypes.POINTER(ctypes.c_float)
    sig = {
        "fac_last_error": (ctypes.c_char_p, []),
        "fac_ctx_create": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int]),
        "fac_ctx_destroy": (ctypes.c_int, [vp]),
        "fac_add_problem": (ctypes.c_int, [vp, ip, dp, dp, ctypes.c_int, ip, ip, ip, ip]),
        "fac_set_coarse_extension": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_set_bc_faces": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]),
        "fac_set_wait_test": (ctypes.c_int, [vp, ctypes.c_longlong, ctypes.c_int]),
        "fac_clear_device_error": (ctypes.c_int, [vp]),
        "fac_fill_table": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_longlong),
                                          ctypes.POINTER(ctypes.c_longlong), ctypes.c_size_t,
                                          szp]),
        "fac_vec_dot": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, dp]),
        "fac_vec_l2_norm": (ctypes.c_int, [vp, ctypes.c_int, dp]),
        "fac_vec_max_norm": (ctypes.c_int, [vp, ctypes.c_int, dp]),
        "fac_vec_linear_sum": (ctypes.c_int, [vp, ctypes.c_int, dp, ctypes.c_int, dp,
                                              ctypes.c_int]),
        "fac_extend_coefficients": (ctypes.c_int, [vp]),
        "fac_tag_gradient": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                            ctypes.POINTER(ctypes.c_longlong)]),
        "fac_download_tags": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, vp]),
        "fac_cluster_tags": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip, ip,
                                            ip, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                            ip, ip]),
        "fac_cluster_tags_all": (ctypes.c_int, [vp, ctypes.c_int, ip, ip, ip, ip, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_int, ip, ip]),
        "fac_set_poisson": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_double]),
        "fac_set_bc": (ctypes.c_int, [vp, dp, dp, dp]),
        "fac_set_params": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_int, ctypes.c_int]),
        "fac_initialize": (ctypes.c_int, [vp]),
        "fac_set_precision": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_set_graph": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_set_fused": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_set_staged": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_solve_fgmres": (ctypes.c_int, [vp, ctypes.c_int, ip, ip, dp]),
        "fac_set_krylov": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_set_learned": (ctypes.c_int, [vp, vp, ctypes.c_int]),
        "fac_learned_samples": (ctypes.c_int, [vp, ctypes.c_int, vp, dp]),
        "fac_set_fused_residual": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_set_stage_budget": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_set_stage_depth": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_autotune": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int), dp]),
        "fac_field_size": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, szp]),
        "fac_side_size": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, szp]),
        "fac_oside_size": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, szp]),
        "fac_upload_field": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]),
        "fac_download_field": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]),
        "fac_upload_side": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, dp]),
        "fac_download_side": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, dp]),
        "fac_download_flux": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, dp]),
        "fac_download_oside": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, dp]),
        "fac_ghost_fill": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int]),
        "fac_smooth": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, ip]),
        "fac_comp_residual": (ctypes.c_int, [vp] + [ctypes.c_int] * 5),
        "fac_restrict": (ctypes.c_int, [vp] + [ctypes.c_int] * 3),
        "fac_restrict_solution": (ctypes.c_int, [vp] + [ctypes.c_int] * 2),
        "fac_prolong_correct": (ctypes.c_int, [vp] + [ctypes.c_int] * 3),
        "fac_compute_weights": (ctypes.c_int, [vp]),
        "fac_rms_norm": (ctypes.c_int, [vp, ctypes.c_int, dp]),
        "fac_solve_coarsest": (ctypes.c_int, [vp, ip]),
        "fac_fac_cycle": (ctypes.c_int, [vp]),
        "fac_solve": (ctypes.c_int, [vp, ip, ip, dp]),
        "fac_solve_host": (ctypes.c_int, [vp, ctypes.POINTER(dp), ctypes.POINTER(dp),
                                          ctypes.POINTER(dp), ip, ip, dp]),
        "fac_residual_history": (ctypes.c_int, [vp, ctypes.c_int, dp, ctypes.c_int, ip]),
        "fac_coarse_sweeps": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_longlong)]),
        "fac_reset_stats": (ctypes.c_int, [vp]),
        "fac_synchronize": (ctypes.c_int, [vp]),
        "fac_zero_field": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_kernel_launches": (ctypes.c_int, [ctypes.POINTER(ctypes.c_longlong)]),
        "fac_profile_enable": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_profile_read": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong),
                                            dp, dp]),
        "fac_profile_reset": (ctypes.c_int, [vp]),
        "fac_timer": (ctypes.c_int, [vp, ctypes.c_int, dp]),
        "fac_trace_enable": (ctypes.c_int, [vp, ctypes.c_int]),
        "fac_trace_read": (ctypes.c_int, [vp, ctypes.c_char_p, ctypes.c_int, ip]),
        "fac_cnn_last_error": (ctypes.c_char_p, []),
        "fac_cnn_create": (ctypes.c_int, [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int,
                                          ctypes.c_ulonglong]),
        "fac_cnn_destroy": (ctypes.c_int, [vp]),
        "fac_cnn_set_weights": (ctypes.c_int, [vp, fp, fp, fp, fp]),
        "fac_cnn_get_weights": (ctypes.c_int, [vp, fp, fp, fp, fp]),
        "fac_cnn_forward": (ctypes.c_int, [vp, vp, ctypes.c_longlong, vp]),
        "fac_cnn_gradients": (ctypes.c_int, [vp, vp, vp, vp, ctypes.c_longlong, dp, fp, fp,
                                             fp, fp]),
        "fac_cnn_train_step": (ctypes.c_int, [vp, vp, vp, vp, ctypes.c_longlong,
                                              ctypes.c_double, ctypes.c_float, dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def exported_symbols():
    """Names of the C ABI entry points this binding expects."""
    load_library()
    return [n for n in dir(_lib) if n.startswith("fac_")]


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _check(rc):
    if rc != 0:
        raise FacError(rc, load_library().fac_last_error().decode())


class FacContext:
    """A batch of FAC problems on one GPU (device=-1: host-only table check)."""

    def __init__(self, problems: Sequence, params: Optional[dict] = None, device: int = 0,
                 bc=None, precision: str = "fp64", coarse_extension: int = 0):
        L = load_library()
        problems = list(problems)
        if not problems:
            raise ValueError("no problems")
        self.problems = problems
        self.dim = problems[0].dim
        # fac_set_coarse_extension: the library adds this many coarser
        # levels; level numbers below count them
        self.ext = int(coarse_extension)
        self.nlev = problems[0].nlev + self.ext
        self.device = device
        self.stage_depth = 2
        h = ctypes.c_void_p()
        _check(L.fac_ctx_create(ctypes.byref(h), self.dim, device))
        self.h = h
        p0 = problems[0]
        _check(L.fac_set_poisson(h, int(p0.d_variable), float(p0.d_const), int(p0.c_kind),
                                 float(p0.c_const)))
        if bc is not None:
            a, b, g = (np.ascontiguousarray(x, dtype=np.float64) for x in bc)
            _check(L.fac_set_bc(h, _dp(a), _dp(b), _dp(g)))
        prm = dict(max_cycles=100, residual_tol=1e-300, relative_residual_tol=1e-10,
                   pre_sweeps=2, post_sweeps=2, coarse_tol=1e-8, coarse_max_it=500, ewing=1)
        if params:
            prm.update(params)
        self.params = prm
        _check(L.fac_set_params(h, prm["max_cycles"], prm["residual_tol"],
                                prm["relative_residual_tol"], prm["pre_sweeps"],
                                prm["post_sweeps"], prm["coarse_tol"], prm["coarse_max_it"],
                                prm["ewing"]))
        if self.ext:
            _check(L.fac_set_coarse_extension(h, self.ext))
        for prob in problems:
            n0 = np.array(prob.n0, dtype=np.int32)
            xlo = np.array(prob.xlo, dtype=np.float64)
            xup = np.array(prob.xup, dtype=np.float64)
            ratio = np.array([lv.ratio for lv in prob.levels], dtype=np.int32).reshape(-1)
            npatch = np.array([len(lv.boxes) for lv in prob.levels], dtype=np.int32)
            boxes = np.ascontiguousarray(
                np.concatenate([lv.boxes for lv in prob.levels]).astype(np.int32).reshape(-1))
            idx = ctypes.c_int(0)
            _check(L.fac_add_problem(h, _ip(n0), _dp(xlo), _dp(xup), prob.nlev, _ip(ratio),
                                     _ip(npatch), _ip(boxes), ctypes.byref(idx)))
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision = precision
        _check(L.fac_set_precision(h, 1 if precision == "mixed" else 0))
        _check(L.fac_initialize(h))
        if device >= 0:
            for ip_, prob in enumerate(problems):
                for pl in range(prob.nlev):
                    ln = pl + self.ext
                    if prob.f:
                        self.upload(F, ip_, ln, prob.f[pl])
                    if prob.u0:
                        self.upload(U, ip_, ln, prob.u0[pl])
                    if prob.d_variable:
                        self.upload_side(ip_, ln, prob.d[pl])
                    if prob.c_kind == 2:
                        self.upload(C, ip_, ln, prob.c[pl])

    def close(self):
        if getattr(self, "h", None):
            load_library().fac_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nprob(self):
        return len(self.problems)

    # sizes and transfers ----------------------------------------------------
    def size(self, fid, prob, ln):
        n = ctypes.c_size_t(0)
        _check(load_library().fac_field_size(self.h, fid, prob, ln, ctypes.byref(n)))
        return n.value

    def upload(self, fid, prob, ln, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        if arr.size != self.size(fid, prob, ln):
            raise ValueError(f"size {arr.size} != {self.size(fid, prob, ln)}")
        _check(load_library().fac_upload_field(self.h, fid, prob, ln, _dp(arr)))

    def download(self, fid, prob, ln):
        out = np.empty(self.size(fid, prob, ln))
        _check(load_library().fac_download_field(self.h, fid, prob, ln, _dp(out)))
        return out

    def upload_side(self, prob, ln, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        _check(load_library().fac_upload_side(self.h, prob, ln, _dp(arr)))

    def download_side(self, prob, ln):
        out = np.empty(self._side_n(prob, ln))
        _check(load_library().fac_download_side(self.h, prob, ln, _dp(out)))
        return out

    def _side_n(self, prob, ln):
        n = ctypes.c_size_t(0)
        _check(load_library().fac_side_size(self.h, prob, ln, ctypes.byref(n)))
        return n.value

    def download_flux(self, prob, ln):
        out = np.empty(self._side_n(prob, ln))
        _check(load_library().fac_download_flux(self.h, prob, ln, _dp(out)))
        return out

    def download_oside(self, prob, ln):
        n = ctypes.c_size_t(0)
        _check(load_library().fac_oside_size(self.h, prob, ln, ctypes.byref(n)))
        out = np.empty(n.value)
        _check(load_library().fac_download_oside(self.h, prob, ln, _dp(out)))
        return out

    # operators --------------------------------------------------------------
    def ghost_fill(self, fid, ln, with_coarse, homogeneous):
        _check(load_library().fac_ghost_fill(self.h, fid, ln, int(with_coarse), int(homogeneous)))

    def smooth(self, fid_e, fid_r, ln, nsweeps, tol=-1.0):
        sw = np.zeros(self.nprob, dtype=np.int32)
        _check(load_library().fac_smooth(self.h, fid_e, fid_r, ln, nsweeps, tol, _ip(sw)))
        return sw

    def comp_residual(self, fid_r, fid_u, fid_f, ln, error_eq):
        _check(load_library().fac_comp_residual(self.h, fid_r, fid_u, fid_f, ln, int(error_eq)))

    def restrict(self, fid_src, fid_dst, dest_ln):
        _check(load_library().fac_restrict(self.h, fid_src, fid_dst, dest_ln))

    def restrict_solution(self, fid, dest_ln):
        _check(load_library().fac_restrict_solution(self.h, fid, dest_ln))

    def prolong_correct(self, fid_src, fid_dst, dest_ln):
        _check(load_library().fac_prolong_correct(self.h, fid_src, fid_dst, dest_ln))

    def compute_weights(self):
        _check(load_library().fac_compute_weights(self.h))

    def rms_norm(self, fid):
        out = np.zeros(self.nprob)
        _check(load_library().fac_rms_norm(self.h, fid, _dp(out)))
        return out

    def solve_coarsest(self):
        sw = np.zeros(self.nprob, dtype=np.int32)
        _check(load_library().fac_solve_coarsest(self.h, _ip(sw)))
        return sw

    def fac_cycle(self):
        _check(load_library().fac_fac_cycle(self.h))

    def solve(self):
        conv = np.zeros(self.nprob, dtype=np.int32)
        its = np.zeros(self.nprob, dtype=np.int32)
        res = np.zeros(self.nprob)
        _check(load_library().fac_solve(self.h, _ip(conv), _ip(its), _dp(res)))
        return conv.astype(bool), its, res

    def solve_host(self, f_arrays, u_out, u0_arrays=None):
        """End-to-end solve from host buffers (one per problem x level of the
        caller's hierarchy, without the levels of the coarse extension)."""
        n = self.nprob * (self.nlev - self.ext)
        DP = ctypes.POINTER(ctypes.c_double)
        ftab = (DP * n)(*[_dp(a) for a in f_arrays])
        utab = (DP * n)(*[_dp(a) for a in u_out])
        u0tab = (DP * n)(*[_dp(a) for a in u0_arrays]) if u0_arrays is not None else None
        conv = np.zeros(self.nprob, dtype=np.int32)
        its = np.zeros(self.nprob, dtype=np.int32)
        res = np.zeros(self.nprob)
        _check(load_library().fac_solve_host(self.h, ftab, u0tab, utab, _ip(conv), _ip(its),
                                             _dp(res)))
        return conv.astype(bool), its, res

    def residual_history(self, prob):
        cap = self.params["max_cycles"] + 1
        out = np.zeros(cap)
        n = ctypes.c_int(0)
        _check(load_library().fac_residual_history(self.h, prob, _dp(out), cap, ctypes.byref(n)))
        return out[:min(n.value, cap)]

    def coarse_sweeps(self):
        out = np.zeros(self.nprob, dtype=np.int64)
        _check(load_library().fac_coarse_sweeps(
            self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))))
        return out

    def synchronize(self):
        _check(load_library().fac_synchronize(self.h))

    def autotune(self):
        """Pick the staged pass's stage size and depth by timing (before a
        solve); returns (chosen bytes, ms per candidate) with the candidates
        of depth 2 then depth 3; the depth is in stage_depth."""
        chosen = ctypes.c_int(0)
        depth = ctypes.c_int(0)
        ms = np.zeros(10)
        _check(load_library().fac_autotune(self.h, ctypes.byref(chosen), ctypes.byref(depth),
                                           _dp(ms)))
        self.stage_depth = depth.value
        return chosen.value, ms

    def set_stage_budget(self, nbytes):
        _check(load_library().fac_set_stage_budget(self.h, int(nbytes)))

    def set_stage_depth(self, depth):
        _check(load_library().fac_set_stage_depth(self.h, int(depth)))
        self.stage_depth = int(depth)

    def set_fused_residual(self, on=True):
        """One-pass composite residual: True on every level, False on none,
        -1 (the default) on the levels of large patches."""
        _check(load_library().fac_set_fused_residual(self.h, int(on)))

    def set_learned(self, net, level):
        """Apply the learned correction of `net` (a CNN, or None) on `level`
        after every cycle of solve()."""
        _check(load_library().fac_set_learned(self.h, net.h if net is not None else None,
                                              int(level)))
        self._net = net  # keep the network alive while the context uses it

    def learned_samples(self, level, x_ptr, npatch):
        """Network inputs for the current residual of `level` into the device
        array at x_ptr (npatch * CNN_BOX^3 FP32); returns the patch scales."""
        scale = np.zeros(max(1, npatch))
        _check(load_library().fac_learned_samples(self.h, int(level), x_ptr, _dp(scale)))
        return scale[:npatch]

    def set_krylov(self, restart):
        """restart > 0: solve() / solve_host() run FGMRES(restart) around the
        FAC cycle; 0: the stationary FAC iteration."""
        _check(load_library().fac_set_krylov(self.h, int(restart)))

    def solve_fgmres(self, restart=20):
        """FGMRES(restart) with the FAC cycle as preconditioner; same
        outputs as solve()."""
        conv = np.zeros(self.nprob, dtype=np.int32)
        its = np.zeros(self.nprob, dtype=np.int32)
        res = np.zeros(self.nprob)
        _check(load_library().fac_solve_fgmres(self.h, int(restart), _ip(conv), _ip(its),
                                               _dp(res)))
        return conv.astype(bool), its, res

    def set_staged(self, on=True):
        _check(load_library().fac_set_staged(self.h, int(on)))

    def set_fused(self, on=True):
        _check(load_library().fac_set_fused(self.h, int(on)))

    def set_graph(self, on=True):
        _check(load_library().fac_set_graph(self.h, int(on)))

    def zero(self, fid):
        _check(load_library().fac_zero_field(self.h, fid))

    def set_params(self, **changes):
        """Change solver parameters (same keys as the constructor's params)."""
        self.params.update(changes)
        prm = self.params
        _check(load_library().fac_set_params(
            self.h, prm["max_cycles"], prm["residual_tol"], prm["relative_residual_tol"],
            prm["pre_sweeps"], prm["post_sweeps"], prm["coarse_tol"], prm["coarse_max_it"],
            prm["ewing"]))

    def profile(self, on=True):
        _check(load_library().fac_profile_enable(self.h, int(on)))

    def profile_read(self, kind):
        n = ctypes.c_longlong(0)
        ms = ctypes.c_double(0.0)
        by = ctypes.c_double(0.0)
        _check(load_library().fac_profile_read(self.h, kind, ctypes.byref(n), ctypes.byref(ms),
                                               ctypes.byref(by)))
        return n.value, ms.value, by.value

    def trace(self, on=True):
        _check(load_library().fac_trace_enable(self.h, int(on)))

    def trace_read(self):
        import json
        n = ctypes.c_int(0)
        _check(load_library().fac_trace_read(self.h, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value + 1)
        _check(load_library().fac_trace_read(self.h, buf, n.value + 1, ctypes.byref(n)))
        return json.loads(buf.value.decode())

    def set_bc_faces(self, faces, prob=0):
        """Robin coefficients varying along the boundary: {(level,
        location): (n, 3) array of (a, b, g)} over each level's domain face
        (fac_set_bc_faces); levels count the coarse extension's."""
        for (ln, loc), abg in faces.items():
            arr = np.ascontiguousarray(abg, dtype=np.float64).reshape(-1)
            _check(load_library().fac_set_bc_faces(self.h, prob, int(ln), int(loc), _dp(arr)))

    def fill_table(self, ln, with_coarse):
        """(dst, src) element copies of a ghost fill of level ln
        (fac_fill_table); src < 0 is element -src-1 of the coarser level."""
        L = load_library()
        n = ctypes.c_size_t(0)
        _check(L.fac_fill_table(self.h, ln, int(with_coarse), None, None, 0, ctypes.byref(n)))
        dst = np.zeros(n.value, dtype=np.int64)
        src = np.zeros(n.value, dtype=np.int64)
        lp = ctypes.POINTER(ctypes.c_longlong)
        _check(L.fac_fill_table(self.h, ln, int(with_coarse), dst.ctypes.data_as(lp),
                                src.ctypes.data_as(lp), n.value, ctypes.byref(n)))
        return dst, src

    # composite-vector operations (SAMRAIVectorReal dot, norms, linearSum)
    def vec_dot(self, fx, fy):
        out = np.zeros(self.nprob)
        _check(load_library().fac_vec_dot(self.h, fx, fy, _dp(out)))
        return out

    def vec_l2_norm(self, fid):
        out = np.zeros(self.nprob)
        _check(load_library().fac_vec_l2_norm(self.h, fid, _dp(out)))
        return out

    def vec_max_norm(self, fid):
        out = np.zeros(self.nprob)
        _check(load_library().fac_vec_max_norm(self.h, fid, _dp(out)))
        return out

    def vec_linear_sum(self, fz, a, fx, b, fy):
        a = np.ascontiguousarray(np.broadcast_to(a, self.nprob), dtype=np.float64)
        b = np.ascontiguousarray(np.broadcast_to(b, self.nprob), dtype=np.float64)
        _check(load_library().fac_vec_linear_sum(self.h, fz, _dp(a), fx, _dp(b), fy))

    # regrid step -----------------------------------------------------------
    def tag_gradient(self, fid, ln, threshold):
        """Tag the cells of level ln where the adaption estimate of field
        fid exceeds threshold (fac_tag_gradient); returns the count per
        problem."""
        cnt = np.zeros(self.nprob, dtype=np.int64)
        _check(load_library().fac_tag_gradient(
            self.h, fid, ln, float(threshold), cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))))
        return cnt

    def download_tags(self, prob, ln):
        out = np.empty(self.size(F, prob, ln), dtype=np.uint8)
        _check(load_library().fac_download_tags(self.h, prob, ln, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def cluster_tags(self, prob, ln, bound, min_box, max_box=(0, 0, 0), efficiency=0.8,
                     combine=0.8):
        """Berger-Rigoutsos boxes (n, 6) over the tags of level ln of one
        problem within the bound boxes (fac_cluster_tags)."""
        bound = np.ascontiguousarray(np.asarray(bound, dtype=np.int32).reshape(-1, 6))
        mn = np.ascontiguousarray(list(min_box) + [1] * (3 - len(min_box)), dtype=np.int32)
        mx = np.ascontiguousarray(list(max_box) + [0] * (3 - len(max_box)), dtype=np.int32)
        cap = 1024
        while True:
            out = np.zeros((cap, 6), dtype=np.int32)
            nb = ctypes.c_int(0)
            _check(load_library().fac_cluster_tags(self.h, prob, ln, len(bound), _ip(bound),
                                                   _ip(mn), _ip(mx), float(efficiency),
                                                   float(combine), cap, _ip(out),
                                                   ctypes.byref(nb)))
            if nb.value <= cap:
                return out[:nb.value].copy()
            cap = nb.value

    def cluster_tags_all(self, ln, bounds, min_box, max_box=(0, 0, 0), efficiency=0.8,
                         combine=0.8):
        """cluster_tags for every problem at once (fac_cluster_tags_all):
        bounds[p] are problem p's bound boxes; returns one (n, 6) array of
        boxes per problem."""
        bl = [np.asarray(b, dtype=np.int32).reshape(-1, 6) for b in bounds]
        if len(bl) != self.nprob:
            raise ValueError("one list of bound boxes per problem")
        nbound = np.ascontiguousarray([len(b) for b in bl], dtype=np.int32)
        bound = np.ascontiguousarray(np.concatenate(bl, axis=0))
        mn = np.ascontiguousarray(list(min_box) + [1] * (3 - len(min_box)), dtype=np.int32)
        mx = np.ascontiguousarray(list(max_box) + [0] * (3 - len(max_box)), dtype=np.int32)
        counts = np.zeros(self.nprob, dtype=np.int32)
        cap = 4096
        while True:
            out = np.zeros((cap, 6), dtype=np.int32)
            _check(load_library().fac_cluster_tags_all(self.h, ln, _ip(nbound), _ip(bound),
                                                       _ip(mn), _ip(mx), float(efficiency),
                                                       float(combine), cap, _ip(out),
                                                       _ip(counts)))
            total = int(counts.sum())
            if total <= cap:
                ends = np.cumsum(counts)
                return [out[e - c:e].copy() for c, e in zip(counts, ends)]
            cap = total

    def timer_start(self):
        _check(load_library().fac_timer(self.h, 0, None))

    def timer_stop(self):
        ms = ctypes.c_double(0.0)
        _check(load_library().fac_timer(self.h, 1, ctypes.byref(ms)))
        return ms.value


def kernel_launches():
    n = ctypes.c_longlong(0)
    _check(load_library().fac_kernel_launches(ctypes.byref(n)))
    return n.value


class CellPoissonFACSolver:
    """Drop-in for solv::CellPoissonFACSolver (CellPoissonFACSolver.h:116-475).

    The reference identifies data by patch-data ids on a PatchHierarchy; here
    a :class:`samrai_b200.configs.Problem` carries the hierarchy and its u,
    f, D and C arrays, and the solver writes the converged u back into it.
    Input keys and defaults follow FACPreconditioner (FACPreconditioner.C:
    80-114) and CellPoissonFACOps (CellPoissonFACOps.C:692-739).
    """

    def __init__(self, dim: int, object_name: str = "CellPoissonFACSolver",
                 input_db: Optional[dict] = None):
        self.dim = dim
        self.object_name = object_name
        db = dict(input_db or {})
        self._params = dict(max_cycles=db.get("max_cycles", 10),
                            residual_tol=db.get("residual_tol", 1e-6),
                            relative_residual_tol=db.get("relative_residual_tol", -1.0),
                            pre_sweeps=db.get("num_pre_sweeps", 1),
                            post_sweeps=db.get("num_post_sweeps", 1),
                            coarse_tol=db.get("coarse_solver_tolerance", 1e-8),
                            coarse_max_it=db.get("coarse_solver_max_iterations", 500),
                            ewing=1)
        if db.get("coarse_solver_choice", "redblack") not in ("redblack", "jacobi"):
            raise ValueError("coarse_solver_choice must be redblack (hypre is not built)")
        if db.get("cf_discretization", "Ewing") != "Ewing":
            raise ValueError("only cf_discretization = Ewing is implemented")
        if db.get("prolongation_method", "LINEAR_REFINE") != "LINEAR_REFINE":
            raise ValueError("only prolongation_method = LINEAR_REFINE is implemented")
        self._d_const = 1.0
        self._d_variable = False
        self._c_kind = 0
        self._c_const = 0.0
        self._bc = None
        self._ctx: Optional[FacContext] = None
        self._problems = None
        self._device = 0
        self._last = None

    # PoissonSpecifications setters (CellPoissonFACSolver.h:312-365)
    def setDConstant(self, d):
        self._d_const, self._d_variable = float(d), False

    def setDPatchDataId(self, flag=True):
        self._d_variable = True

    def setCConstant(self, c):
        self._c_kind, self._c_const = (0, 0.0) if c == 0 else (1, float(c))

    def setCPatchDataId(self, flag=True):
        self._c_kind = 2

    def setBoundaries(self, boundary_type="Dirichlet"):
        """setBoundaries (CellPoissonFACSolver.h:264): only Dirichlet with
        the cached ghost value g=0 or Robin coefficient triples."""
        if boundary_type != "Dirichlet":
            raise ValueError("only Dirichlet boundaries are supported here")
        self._bc = None

    def setBcObject(self, a, b, g):
        self._bc = (a, b, g)

    def setBcFaces(self, faces):
        """Robin coefficients varying along the boundary, {(level,
        location): (n, 3) array of (a, b, g) over the level's domain face}:
        what a RobinBcCoefStrategy's setBcCoefs would fill, evaluated on
        every boundary face."""
        self._faces = dict(faces)

    def setMaxCycles(self, n):
        self._params["max_cycles"] = int(n)

    def setResidualTolerance(self, tol, relative_tol=-1.0):
        self._params["residual_tol"] = float(tol)
        self._params["relative_residual_tol"] = float(relative_tol)

    def setPresmoothingSweeps(self, n):
        self._params["pre_sweeps"] = int(n)

    def setPostsmoothingSweeps(self, n):
        self._params["post_sweeps"] = int(n)

    def setCoarsestLevelSolverTolerance(self, tol):
        self._params["coarse_tol"] = float(tol)

    def setCoarsestLevelSolverMaxIterations(self, n):
        self._params["coarse_max_it"] = int(n)

    def initializeSolverState(self, problems, device: int = 0):
        """initializeSolverState (CellPoissonFACSolver.h:402): builds the
        device state for one problem or a batch of problems."""
        if not isinstance(problems, (list, tuple)):
            problems = [problems]
        for p in problems:
            p.d_variable, p.d_const = self._d_variable or p.d_variable, self._d_const
            if self._c_kind:
                p.c_kind, p.c_const = self._c_kind, self._c_const
        self._problems = list(problems)
        self._ctx = FacContext(self._problems, self._params, device=device, bc=self._bc)
        if getattr(self, "_faces", None):
            for i in range(len(self._problems)):
                self._ctx.set_bc_faces(self._faces, prob=i)

    def deallocateSolverState(self):
        if self._ctx:
            self._ctx.close()
        self._ctx = None

    def solveSystem(self, problems=None):
        """solveSystem (CellPoissonFACSolver.h:183/214).  Returns True when
        every problem converged; the solution is stored in each problem's
        ``u`` list."""
        own = self._ctx is None
        if own:
            self.initializeSolverState(problems)
        conv, its, res = self._ctx.solve()
        for ip_, p in enumerate(self._problems):
            p.u = [self._ctx.download(U, ip_, ln) for ln in range(p.nlev)]
        self._last = (conv, its, res)
        if own:
            self.deallocateSolverState()
        return bool(conv.all())

    def getNumberOfIterations(self):
        return int(self._last[1].max())

    def getResidualNorm(self):
        return float(self._last[2].max())

    def getConvergenceFactors(self):
        hist = self._ctx.residual_history(0) if self._ctx else None
        if hist is None or len(hist) < 2:
            return float("nan"), float("nan")
        net = hist[-1] / (hist[0] + 1e-20)
        avg = net ** (1.0 / (len(hist) - 1))
        return avg, hist[-1] / hist[-2]


CNN_BOX = 18
CNN_SHAPES = [(27, 16), (27, 16, 16), (27, 16, 16), (27, 16)]


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _cnn_check(rc):
    if rc != 0:
        raise FacError(rc, load_library().fac_cnn_last_error().decode())


class CNN:
    """The learned coarse-correction network (fac_cnn_* in the C ABI).
    Inputs and outputs are device pointers (e.g. torch CUDA tensors'
    data_ptr()) holding nsamp * 18^3 FP32 values."""

    def __init__(self, max_batch, device=0, seed=0):
        self.h = ctypes.c_void_p()
        _cnn_check(load_library().fac_cnn_create(ctypes.byref(self.h), device, max_batch, seed))
        self.max_batch = max_batch

    def close(self):
        if getattr(self, "h", None):
            load_library().fac_cnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_weights(self, ws):
        ws = [np.ascontiguousarray(w, dtype=np.float32).reshape(s) for w, s in zip(ws, CNN_SHAPES)]
        _cnn_check(load_library().fac_cnn_set_weights(self.h, *[_fp(w) for w in ws]))

    def get_weights(self):
        ws = [np.zeros(s, dtype=np.float32) for s in CNN_SHAPES]
        _cnn_check(load_library().fac_cnn_get_weights(self.h, *[_fp(w) for w in ws]))
        return ws

    def forward(self, x_ptr, nsamp, y_ptr):
        _cnn_check(load_library().fac_cnn_forward(self.h, x_ptr, nsamp, y_ptr))

    def gradients(self, x_ptr, t_ptr, m_ptr, nsamp):
        gs = [np.zeros(s, dtype=np.float32) for s in CNN_SHAPES]
        loss = ctypes.c_double(0.0)
        _cnn_check(load_library().fac_cnn_gradients(self.h, x_ptr, t_ptr, m_ptr, nsamp,
                                                    ctypes.byref(loss), *[_fp(g) for g in gs]))
        return loss.value, gs

    def train_step(self, x_ptr, t_ptr, m_ptr, nsamp, mask_sum, lr):
        loss = ctypes.c_double(0.0)
        _cnn_check(load_library().fac_cnn_train_step(self.h, x_ptr, t_ptr, m_ptr, nsamp,
                                                     float(mask_sum), float(lr),
                                                     ctypes.byref(loss)))
        return loss.value
