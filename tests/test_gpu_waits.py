"""Bounded device waits.

Every wait of the staged colour pass (a unit's copies landing in shared
memory, a stage coming free) gives up after a bound and sets the context's
device error flag instead of hanging the GPU; the next norm reports
FAC_ERR_CUDA and the context stays usable.  Here the consumer warps are made
to wait on an mbarrier nothing arrives on, with a 1e6-cycle bound: the pass
must end with the error, and after the flag is cleared the same context must
smooth exactly like the oracle again.
"""
import numpy as np
import pytest

from samrai_b200 import configs, fac
from oracle.oracle import E, Oracle, R

pytestmark = pytest.mark.gpu

FAC_ERR_CUDA = 3


def test_bounded_wait_runs_out_and_context_recovers(require_gpu):
    p = configs.small_3d(seed=7)
    prm = dict(coarse_tol=1e-10, max_cycles=2)
    g = fac.FacContext([p], params=prm)
    o = Oracle(p, params=prm)
    ln = p.nlev - 1
    rng = np.random.default_rng(11)
    vals = {fid: rng.standard_normal(o.size(fid, ln)) for fid in (E, R)}
    for l2 in range(p.nlev):
        for fid in (E, R):
            v = vals[fid] if l2 == ln else np.zeros(o.size(fid, l2))
            g.upload(fid, 0, l2, v)
            o.set(fid, l2, v)
    L = fac.load_library()
    assert L.fac_set_wait_test(g.h, 1_000_000, 1) == 0
    g.smooth(E, R, ln, 1)
    with pytest.raises(fac.FacError) as err:
        g.rms_norm(R)
    assert err.value.code == FAC_ERR_CUDA
    # back to the default bound: the context works and matches the oracle
    assert L.fac_set_wait_test(g.h, 4_000_000_000, 0) == 0
    assert L.fac_clear_device_error(g.h) == 0
    for fid in (E, R):
        g.upload(fid, 0, ln, vals[fid])
    g.smooth(E, R, ln, 2)
    o.smooth(E, R, ln, 2)
    assert np.array_equal(g.download(E, 0, ln), o.get(E, ln))
    g.rms_norm(R)
    g.close()
