"""Linear time interpolation of cell, side, face, node and edge data on the
device (fac_time_interpolate) against the reference's own routines.

oracle/_ref/libref_kernels.so holds the reference's Fortran kernels
(pdat_m4lintimeintops{2,3}d.i, expanded and translated to C by the
reference build); each routine is called the way its
*DoubleLinearTimeInterpolateOp calls it (the centered where box, the data's
cell ghost boxes, tfrac as CellDoubleLinearTimeInterpolateOp.C computes it)
and must give the same array, bit for bit, as one batched device call over
all the boxes.
"""
import ctypes
import os

import numpy as np
import pytest

from samrai_b200 import fac

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libref_kernels.so")
CELL, SIDE, FACE, NODE, EDGE = range(5)
NAMES = {CELL: "cell", SIDE: "side", FACE: "face", NODE: "node", EDGE: "edge"}


class TimeBox(ctypes.Structure):
    _fields_ = [("old_data", ctypes.c_void_p), ("new_data", ctypes.c_void_p),
                ("dst_data", ctypes.c_void_p)] + [
        (n, ctypes.c_int * 3) for n in ("where_lo", "where_hi", "old_lo", "old_hi", "new_lo",
                                        "new_hi", "dst_lo", "dst_hi")]


def centered(L, dim, c, axis, lo, hi):
    lo3 = (ctypes.c_int * 3)(*(list(lo) + [0] * (3 - dim)))
    hi3 = (ctypes.c_int * 3)(*(list(hi) + [0] * (3 - dim)))
    olo, ohi = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
    assert L.fac_centered_box(dim, c, axis, lo3, hi3, olo, ohi) == 0
    return list(olo)[:dim], list(ohi)[:dim]


def cases(dim):
    out = [(CELL, 0)]
    for c in (SIDE, FACE, EDGE):
        out += [(c, a) for a in range(dim)]
    return out + [(NODE, 0)]


@pytest.mark.parametrize("dim", [2, 3])
def test_time_interpolation_matches_reference_routines(dim, require_gpu):
    import torch
    if not os.path.exists(REF):
        pytest.skip("the reference build (oracle/_ref) is absent")
    ref = ctypes.CDLL(REF)
    L = fac.load_library()
    L.fac_time_interpolate.argtypes = [ctypes.c_int, ctypes.POINTER(TimeBox), ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_void_p]
    rng = np.random.default_rng(dim)
    # cell ghost boxes of the three data and the cell where box inside all
    patch_lo, patch_hi = np.array([3, -2, 5][:dim]), np.array([14, 9, 13][:dim])
    ghosts = {"old": 1, "new": 2, "dst": 1}
    gbox = {k: (patch_lo - g, patch_hi + g) for k, g in ghosts.items()}
    where = (patch_lo - 1, patch_hi + 1)
    t_old, t_new, t_dst = 0.25, 1.0, 0.6
    tfrac = (t_dst - t_old) / (t_new - t_old)
    boxes, arrays, wants = [], [], []
    for c, axis in cases(dim):
        arr = {}
        for k in ("old", "new", "dst"):
            blo, bhi = centered(L, dim, c, axis, *gbox[k])
            n = int(np.prod(np.asarray(bhi) - np.asarray(blo) + 1))
            arr[k] = (blo, bhi, rng.standard_normal(n))
        wlo, whi = centered(L, dim, c, axis, *where)
        # the reference routine, called as its operator calls it
        want = arr["dst"][2].copy()
        fn = getattr(ref, f"lintimeint{NAMES[c]}doub{dim}d" +
                     (str(axis) if c in (SIDE, FACE, EDGE) else "") + "_")
        ints = [*wlo, *whi]
        for k in ("old", "new", "dst"):
            ints += [int(x) for x in gbox[k][0]] + [int(x) for x in gbox[k][1]]
        iargs = [ctypes.byref(ctypes.c_int(v)) for v in ints]
        dp = ctypes.POINTER(ctypes.c_double)
        fn(*iargs, ctypes.byref(ctypes.c_double(tfrac)),
           arr["old"][2].ctypes.data_as(dp), arr["new"][2].ctypes.data_as(dp),
           want.ctypes.data_as(dp))
        wants.append(want)
        dev = {k: torch.from_numpy(v[2]).cuda() for k, v in arr.items()}
        arrays.append(dev)
        tb = TimeBox()
        tb.old_data, tb.new_data, tb.dst_data = (dev["old"].data_ptr(), dev["new"].data_ptr(),
                                                 dev["dst"].data_ptr())
        pad = lambda v: list(v) + [0] * (3 - dim)
        tb.where_lo[:], tb.where_hi[:] = pad(wlo), pad(whi)
        for k in ("old", "new", "dst"):
            getattr(tb, f"{k}_lo")[:] = pad(arr[k][0])
            getattr(tb, f"{k}_hi")[:] = pad(arr[k][1])
        boxes.append(tb)
    table = (TimeBox * len(boxes))(*boxes)
    assert L.fac_time_interpolate(dim, table, len(boxes), t_old, t_new, t_dst, None) == 0
    torch.cuda.synchronize()
    for (c, axis), dev, want in zip(cases(dim), arrays, wants):
        assert np.array_equal(dev["dst"].cpu().numpy(), want), (NAMES[c], axis)
    # a where box outside an array is refused before anything runs
    bad = TimeBox.from_buffer_copy(boxes[0])
    bad.where_hi[0] += 5
    assert L.fac_time_interpolate(dim, ctypes.byref(bad), 1, t_old, t_new, t_dst, None) == 1
