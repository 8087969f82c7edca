"""Mixed-precision FAC (FP32 smoothing and error transfer, FP64 composite
residual, flux sums, coarsest solve and outer loop): it must reach the same
1e-10 relative residual as FP64 and a converged solution within 1e-9
relative L2 of the FP64 oracle."""
import numpy as np
import pytest

from samrai_b200 import configs, fac
from oracle.oracle import Oracle, U

pytestmark = pytest.mark.gpu


def rel_l2(g, o, nlev, k=0, idx=0):
    """Relative L2 difference over the original levels (offset k)."""
    num = den = 0.0
    for ln in range(nlev):
        a = g.download(U, idx, ln + k)
        b = o.get(U, ln + k)
        num += float(np.sum((a - b) ** 2))
        den += float(np.sum(b ** 2))
    return (num / den) ** 0.5


@pytest.mark.parametrize("mk,mg", [(configs.config1, True), (configs.config3, True),
                                   (configs.small_3d, True), (configs.config1, False)])
def test_mixed_reaches_fp64_accuracy(mk, mg, require_gpu):
    p = mk()
    x = configs.extend_hierarchy(p, min_cells=8 if p.dim == 2 else 4) if mg else p
    k = x.nlev - p.nlev
    prm = dict(coarse_tol=1e-300, coarse_max_it=20 if mg else 500)
    g = fac.FacContext([x], params=prm, precision="mixed")
    conv, its, res = g.solve()
    assert conv[0], (its, res)
    hist = g.residual_history(0)
    assert hist[-1] <= 1e-10 * hist[0] * 1.0000001
    # FP64 oracle solution of the same discrete problem (tight tolerance)
    o = Oracle(x, params=dict(prm, relative_residual_tol=1e-12, max_cycles=200))
    assert o.solve()[0]
    assert rel_l2(g, o, p.nlev, k=k) <= 1e-9


def test_mixed_batched_config5_like(require_gpu):
    probs = [configs.extend_hierarchy(configs.small_3d(seed=s), k=2) for s in (21, 22)]
    prm = dict(coarse_tol=1e-300, coarse_max_it=20)
    g64 = fac.FacContext(probs, params=prm)
    c64, i64, r64 = g64.solve()
    g32 = fac.FacContext(probs, params=prm, precision="mixed")
    c32, i32, r32 = g32.solve()
    assert c64.all() and c32.all()
    # FP32 smoothing costs at most a couple of extra cycles
    assert (i32 <= i64 + 3).all(), (i32, i64)
    for i, p in enumerate(probs):
        num = den = 0.0
        for ln in range(p.nlev):
            a = g32.download(U, i, ln)
            b = g64.download(U, i, ln)
            num += float(np.sum((a - b) ** 2))
            den += float(np.sum(b ** 2))
        assert (num / den) ** 0.5 <= 1e-9
