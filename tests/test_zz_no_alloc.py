"""fac_rms_norm_noalloc: the weighted RMS norm for callers that cannot
allocate device memory (a pool allocator owns all of it, or the call sits
inside a CUDA graph capture).  Its partial sums live in a static device
array instead of context scratch; here it must agree with fac_rms_norm on
the same data, on two calls in a row (the second call reuses the array the
first one left behind).  Kept in its own file, collected last."""
import ctypes

import numpy as np
import pytest

from samrai_b200 import configs, fac

pytestmark = pytest.mark.gpu


def _single_level_problem(n, seed):
    lev0 = configs.Level((1, 1, 1), configs._chop_uniform([n, n, n], 16, 3))
    p = configs.Problem(dim=3, n0=(n, n, n), xlo=(0, 0, 0), xup=(1, 1, 1), levels=[lev0])
    p.f = [np.zeros(configs.field_size(p, 0, 0))]
    p.u0 = [np.zeros(configs.field_size(p, 0, 1))]
    return p


def test_no_alloc_norm_matches_context_norm(require_gpu):
    import torch

    lib = fac.load_library()
    lib.fac_rms_norm_noalloc.restype = ctypes.c_int
    lib.fac_rms_norm_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.POINTER(ctypes.c_longlong), ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p]
    probs = [_single_level_problem(n, s) for s, n in enumerate((16, 32, 48))]
    ctx = fac.FacContext(probs)
    rng = np.random.default_rng(7)
    xs, ws = [], []
    for i in range(len(probs)):
        r = rng.standard_normal(ctx.size(fac.R, i, 0))
        ctx.upload(fac.R, i, 0, r)
        xs.append(r)
        ws.append(ctx.download(fac.W, i, 0))
    want = ctx.rms_norm(fac.R)

    x = torch.from_numpy(np.concatenate(xs)).cuda()
    w = torch.from_numpy(np.concatenate(ws)).cuda()
    offs = np.concatenate([[0], np.cumsum([a.size for a in xs])]).astype(np.int64)
    off_p = offs.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out = torch.full((len(probs),), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.fac_rms_norm_noalloc(x.data_ptr(), w.data_ptr(), off_p, len(probs),
                                      out.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=1e-13, atol=0)

    # sizes beyond the static array are rejected, not truncated
    big = np.zeros(258, dtype=np.int64)
    rc = lib.fac_rms_norm_noalloc(x.data_ptr(), w.data_ptr(),
                                  big.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), 257,
                                  out.data_ptr(), stream)
    assert rc == 1
    ctx.close()
