"""fac_rms_norm_noalloc: the weighted RMS norm for callers that cannot
allocate device memory when they need a norm (all device memory handed to a
pool allocator up front, or a time step that may not call cudaMalloc because
it synchronises the device).  Its partial sums live in a static device array
instead of context scratch.  Here it must agree with fac_rms_norm on the
same data on two calls in a row (the second call reuses the array the first
one left behind), leave the device's free memory unchanged, give 0 for an
empty segment, accept the full FAC_NOALLOC_MAX_SEGMENTS segments and reject
one more.  Kept in its own file, collected last."""
import ctypes

import numpy as np
import pytest

from samrai_b200 import configs, fac

pytestmark = pytest.mark.gpu

MAX_SEGMENTS = 256  # FAC_NOALLOC_MAX_SEGMENTS


def _single_level_problem(n, seed):
    lev0 = configs.Level((1, 1, 1), configs._chop_uniform([n, n, n], 16, 3))
    p = configs.Problem(dim=3, n0=(n, n, n), xlo=(0, 0, 0), xup=(1, 1, 1), levels=[lev0])
    p.f = [np.zeros(configs.field_size(p, 0, 0))]
    p.u0 = [np.zeros(configs.field_size(p, 0, 1))]
    return p


def _entry():
    lib = fac.load_library()
    fn = lib.fac_rms_norm_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
                   ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    return fn


def _offsets(offs):
    offs = np.ascontiguousarray(offs, dtype=np.int64)
    return offs, offs.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))


def test_no_alloc_norm_matches_context_norm(require_gpu):
    import torch

    norm = _entry()
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
    offs, off_p = _offsets(np.concatenate([[0], np.cumsum([a.size for a in xs])]))
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((MAX_SEGMENTS,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    def call():
        out.fill_(float("nan"))
        rc = norm(x.data_ptr(), w.data_ptr(), off_p, len(probs), out.data_ptr(), stream)
        assert rc == 0
        torch.cuda.synchronize()
        got = out[:len(probs)].cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=1e-13, atol=0)

    # the first calls may load modules (the library's and torch's); after
    # them, ten more calls leave the device's free memory as it was
    for _ in range(3):
        call()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(10):
        call()
    assert torch.cuda.mem_get_info()[0] == free0

    # the full segment count, with empty segments among them: every
    # segment's norm against numpy, an empty one is 0
    cuts = np.sort(rng.integers(0, x.numel(), MAX_SEGMENTS - 1))
    cuts[10] = cuts[11]  # segment 11 is empty
    offs, off_p = _offsets(np.concatenate([[0], cuts, [x.numel()]]))
    rc = norm(x.data_ptr(), w.data_ptr(), off_p, MAX_SEGMENTS, out.data_ptr(), stream)
    assert rc == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    xh, wh = x.cpu().numpy(), w.cpu().numpy()
    for s in range(MAX_SEGMENTS):
        a, b = offs[s], offs[s + 1]
        sw = wh[a:b].sum()
        ref = np.sqrt((xh[a:b] ** 2 * wh[a:b]).sum()) / np.sqrt(sw) if sw > 0 else 0.0
        np.testing.assert_allclose(got[s], ref, rtol=1e-12, atol=0)
    assert got[11] == 0.0

    # one segment beyond the static array is rejected, not truncated
    big, big_p = _offsets(np.zeros(MAX_SEGMENTS + 2))
    rc = norm(x.data_ptr(), w.data_ptr(), big_p, MAX_SEGMENTS + 1, out.data_ptr(), stream)
    assert rc == 1
    ctx.close()
