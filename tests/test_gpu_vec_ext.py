"""Composite-vector operations and the multigrid coarse extension through
the C ABI.

fac_vec_dot / fac_vec_l2_norm / fac_vec_max_norm / fac_vec_linear_sum are
SAMRAIVectorReal's dot, L2Norm, maxNorm and linearSum over a FAC hierarchy
(solv/SAMRAIVectorReal.C:821-960) with the control-volume weights: checked
against numpy on the same data (the dot to 1e-13 relative, the maximum and
the linear sum bit for bit; ghost cells untouched).

fac_set_coarse_extension adds domain-covering coarser levels inside the
library; a solve with it must equal, bit for bit, the solve of the same
hierarchy extended on the host (samrai_b200.configs.extend_hierarchy), and
the derived coefficients on the added levels must be the same numbers.
"""
import numpy as np
import pytest

from samrai_b200 import configs, fac
from oracle.oracle import E, F, R, TR, U, W

pytestmark = pytest.mark.gpu


def _interior(p, ln, arr, g):
    out = []
    for _, _, v in configs.patch_views(p, ln, arr, g):
        if g:
            v = v[1:-1, 1:-1, 1:-1] if p.dim == 3 else v[:, 1:-1, 1:-1]
        out.append(v.reshape(-1))
    return np.concatenate(out)


GHOST = {U: 1, E: 1, F: 0, R: 0, TR: 0}


def test_vector_operations_match_numpy(require_gpu):
    probs = [configs.small_3d(seed=21), configs.small_3d(seed=22)]
    g = fac.FacContext(probs)
    rng = np.random.default_rng(5)
    data = {}
    for fid in (U, E, F, R, TR):
        for i, p in enumerate(probs):
            for ln in range(p.nlev):
                v = rng.standard_normal(g.size(fid, i, ln))
                g.upload(fid, i, ln, v)
                data[fid, i, ln] = v
    w = {(i, ln): g.download(W, i, ln) for i, p in enumerate(probs) for ln in range(p.nlev)}

    def inner(fx, fy, i):
        p = probs[i]
        return sum(float(np.sum(_interior(p, ln, data[fx, i, ln], GHOST[fx]) *
                                _interior(p, ln, data[fy, i, ln], GHOST[fy]) * w[i, ln]))
                   for ln in range(p.nlev))

    for fx, fy in ((U, R), (E, E), (F, TR)):
        got = g.vec_dot(fx, fy)
        for i in range(len(probs)):
            want = inner(fx, fy, i)
            assert abs(got[i] - want) <= 1e-13 * max(abs(want), 1e-300), (fx, fy, i)
    got = g.vec_l2_norm(R)
    for i in range(len(probs)):
        assert abs(got[i] - np.sqrt(inner(R, R, i))) <= 1e-13 * got[i]
    got = g.vec_max_norm(U)
    for i, p in enumerate(probs):
        want = max(float(np.abs(_interior(p, ln, data[U, i, ln], 1)[w[i, ln] > 0]).max())
                   for ln in range(p.nlev) if np.any(w[i, ln] > 0))
        assert got[i] == want

    a, b = np.array([0.75, -1.5]), np.array([2.0, 0.25])
    g.vec_linear_sum(E, a, U, b, R)
    for i, p in enumerate(probs):
        for ln in range(p.nlev):
            z = g.download(E, i, ln)
            want = a[i] * _interior(p, ln, data[U, i, ln], 1) + \
                b[i] * _interior(p, ln, data[R, i, ln], 0)
            assert np.array_equal(_interior(p, ln, z, 1), want), (i, ln)
            # ghost cells keep their values
            m = np.ones(z.size, dtype=bool)
            m[_interior(p, ln, np.arange(z.size), 1)] = False
            assert np.array_equal(z[m], data[E, i, ln][m]), (i, ln)
    g.close()


def _varcoef_3d(seed):
    p = configs.small_3d(seed=seed)
    d = configs.random_field(seed + 3, 3).exp()
    p.d_variable = True
    p.d = [configs.fill_side_field(p, ln, d) for ln in range(p.nlev)]
    return p


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_coarse_extension_in_library_equals_host_extension(precision, require_gpu):
    k = 2
    probs = [_varcoef_3d(31), _varcoef_3d(32)]
    host = [configs.extend_hierarchy(p, k=k) for p in probs]
    prm = dict(coarse_tol=1e-300, coarse_max_it=20, max_cycles=30)
    a = fac.FacContext(host, params=prm, precision=precision)
    b = fac.FacContext(probs, params=prm, precision=precision, coarse_extension=k)
    ca, ia, ra = a.solve()
    cb, ib, rb = b.solve()
    assert np.array_equal(ia, ib) and np.array_equal(ra, rb)
    for i in range(len(probs)):
        assert np.array_equal(a.residual_history(i), b.residual_history(i))
        for ln in range(host[i].nlev):
            assert np.array_equal(a.download(U, i, ln), b.download(U, i, ln)), (i, ln)
            if ln < k:
                assert np.array_equal(b.download_side(i, ln), host[i].d[ln]), (i, ln)
    # end to end from host buffers: the tables hold the caller's levels only
    f_host = [np.ascontiguousarray(p.f[ln]) for p in probs for ln in range(p.nlev)]
    u_host = [np.empty(configs.field_size(p, ln, 1)) for p in probs for ln in range(p.nlev)]
    cc, ic, rc = b.solve_host(f_host, u_host)
    assert np.array_equal(ic, ib)
    for i, p in enumerate(probs):
        for ln in range(p.nlev):
            assert np.array_equal(u_host[i * p.nlev + ln], b.download(U, i, ln + k)), (i, ln)
    a.close()
    b.close()
