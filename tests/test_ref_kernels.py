"""The reference's time-interpolation routines (oracle/_ref/libref_kernels.so,
its Fortran translated to C by the reference build) against a numpy
restatement of what fac_time_interpolate computes: for every centering in
2-D and 3-D, dst = old (1 - t) + new t over the centered where box, each
array indexed in its own centered box, everything else untouched."""
import ctypes
import os

import numpy as np
import pytest

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libref_kernels.so")
CELL, SIDE, FACE, NODE, EDGE = range(5)
NAMES = {CELL: "cell", SIDE: "side", FACE: "face", NODE: "node", EDGE: "edge"}


def centered(dim, c, axis, lo, hi):
    """fac_centered_box restated: the index box of centering c."""
    lo, hi = list(lo), list(hi)
    if c == SIDE:
        hi[axis] += 1
    elif c == NODE:
        hi = [h + 1 for h in hi]
    elif c == EDGE:
        hi = [h + (0 if a == axis else 1) for a, h in enumerate(hi)]
    elif c == FACE:
        order = [(axis + q) % dim for q in range(dim)]
        lo = [lo[y] for y in order]
        hi = [hi[y] + (1 if q == 0 else 0) for q, y in enumerate(order)]
    return lo, hi


def view(a, lo, hi):
    ext = [h - l + 1 for l, h in zip(lo, hi)]
    return a.reshape(ext[::-1])


def region(lo_box, wlo, whi):
    return tuple(slice(wl - bl, wh - bl + 1) for bl, wl, wh in
                 list(zip(lo_box, wlo, whi))[::-1])


@pytest.mark.parametrize("dim", [2, 3])
def test_reference_time_interpolation_is_the_restated_formula(dim):
    if not os.path.exists(REF):
        pytest.skip("the reference build (oracle/_ref) is absent")
    ref = ctypes.CDLL(REF)
    rng = np.random.default_rng(10 + dim)
    plo, phi = np.array([2, -3, 4][:dim]), np.array([9, 6, 11][:dim])
    gbox = {"old": (plo - 1, phi + 1), "new": (plo - 2, phi + 2), "dst": (plo - 1, phi + 1)}
    where = (plo - 1, phi)
    t = (0.7 - 0.2) / (1.3 - 0.2)
    cases = [(CELL, 0)] + [(c, a) for c in (SIDE, FACE, EDGE) for a in range(dim)] + [(NODE, 0)]
    for c, axis in cases:
        arr = {}
        for k, (lo, hi) in gbox.items():
            blo, bhi = centered(dim, c, axis, lo, hi)
            arr[k] = (blo, bhi, rng.standard_normal(int(np.prod(np.subtract(bhi, blo) + 1))))
        wlo, whi = centered(dim, c, axis, *where)
        got = arr["dst"][2].copy()
        fn = getattr(ref, f"lintimeint{NAMES[c]}doub{dim}d" +
                     (str(axis) if c in (SIDE, FACE, EDGE) else "") + "_")
        ints = [*wlo, *whi]
        for k in ("old", "new", "dst"):
            ints += [int(x) for x in gbox[k][0]] + [int(x) for x in gbox[k][1]]
        dp = ctypes.POINTER(ctypes.c_double)
        fn(*[ctypes.byref(ctypes.c_int(v)) for v in ints], ctypes.byref(ctypes.c_double(t)),
           arr["old"][2].ctypes.data_as(dp), arr["new"][2].ctypes.data_as(dp),
           got.ctypes.data_as(dp))
        want = arr["dst"][2].copy()
        w = view(want, *arr["dst"][:2])
        o = view(arr["old"][2], *arr["old"][:2])[region(arr["old"][0], wlo, whi)]
        n = view(arr["new"][2], *arr["new"][:2])[region(arr["new"][0], wlo, whi)]
        w[region(arr["dst"][0], wlo, whi)] = o * (1.0 - t) + n * t
        assert np.array_equal(got, want), (NAMES[c], axis)
