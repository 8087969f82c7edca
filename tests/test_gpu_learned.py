"""Learned coarse correction: training on the GPU with the project's own
CNN kernels on (residual, error) pairs that the FAC solver generates, and
what the trained network gains inside the solve compared with plain FAC."""
import json

import numpy as np
import pytest

from samrai_b200 import configs, fac, learned

PARAMS = dict(max_cycles=100, residual_tol=1e-300, relative_residual_tol=1e-10,
              pre_sweeps=2, post_sweeps=2, coarse_tol=1e-300, coarse_max_it=20, ewing=1)


def _problems(seeds):
    return [configs.extend_hierarchy(configs.config5_problem(s, n0=64), k=3) for s in seeds]


@pytest.mark.gpu
def test_training_lowers_loss_and_correction_never_hurts(require_gpu):
    train = _problems([1000, 1001, 1002, 1003])
    level = train[0].nlev - 1
    pairs = learned.generate_pairs(train, level, [1, 2, 4], params=PARAMS)
    assert pairs.n > 500
    net = fac.CNN(max_batch=2048, seed=3)
    before = learned.masked_loss(net, pairs)
    losses = learned.train(net, pairs, epochs=3, batch=64, lr=1e-3)
    after = learned.masked_loss(net, pairs)
    assert np.isfinite(after) and after < before
    held_out = _problems([2000, 2001])
    ev = learned.evaluate(held_out, level, net, params=PARAMS)
    plain, lrn = ev["plain"], ev["learned"]
    assert plain["converged"].all() and lrn["converged"].all()
    # the minimal-residual step length is 0 whenever the prediction would not
    # lower the residual, so the correction never slows convergence down
    assert (lrn["cycles"] <= plain["cycles"] + 1).all()
    # inside FGMRES(20): the network as the preconditioner's second stage;
    # the flexible method converges whatever the stage returns
    kev = learned.evaluate(held_out, level, net, params=PARAMS, krylov=20)
    kp, kl = kev["plain"], kev["learned"]
    assert kp["converged"].all() and kl["converged"].all()
    gain = {"loss_before": before, "loss_after": after, "epoch_losses": losses,
            "cycles_plain": plain["cycles"].tolist(), "cycles_learned": lrn["cycles"].tolist(),
            "ms_plain": plain["ms"], "ms_learned": lrn["ms"],
            "fgmres_its_plain": kp["cycles"].tolist(), "fgmres_its_learned": kl["cycles"].tolist(),
            "fgmres_ms_plain": kp["ms"], "fgmres_ms_learned": kl["ms"]}
    print(json.dumps(gain))
