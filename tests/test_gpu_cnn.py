"""CUDA kernels of the coarse-correction CNN against the numpy restatement
(oracle/cnn_oracle.py): forward output and all four weight gradients, and a
training run that lowers the loss."""
import numpy as np
import pytest

from samrai_b200 import fac
from oracle import cnn_oracle as co

pytestmark = pytest.mark.gpu

S = fac.CNN_BOX


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-30))


def test_forward_and_gradients_match_oracle(require_gpu):
    import torch
    rng = np.random.default_rng(0)
    n = 2
    ref = co.CNN.init(seed=3)
    x = rng.standard_normal((n, S, S, S)).astype(np.float32)
    t = rng.standard_normal((n, S, S, S)).astype(np.float32)
    mask = np.zeros_like(t)
    mask[:, 1:-1, 1:-1, 1:-1] = 1.0
    net = fac.CNN(max_batch=4)
    net.set_weights(ref.w)
    xd, td, md = (torch.from_numpy(a).cuda() for a in (x, t, mask))
    yd = torch.zeros_like(xd)
    net.forward(xd.data_ptr(), n, yd.data_ptr())
    y_ref, _ = ref.forward(x)
    assert rel(yd.cpu().numpy(), y_ref) < 1e-2
    loss, gs = net.gradients(xd.data_ptr(), td.data_ptr(), md.data_ptr(), n)
    loss_ref, gs_ref = ref.loss_and_grads(x, t, mask)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    for g, gr in zip(gs, gs_ref):
        assert rel(g, gr) < 3e-2, rel(g, gr)
    net.close()


def test_training_lowers_loss(require_gpu):
    import torch
    rng = np.random.default_rng(1)
    n = 8
    # target: a fixed local linear map of the input (a 7-point average)
    x = rng.standard_normal((n, S, S, S)).astype(np.float32)
    t = x.copy()
    for ax in (1, 2, 3):
        t += np.roll(x, 1, axis=ax) + np.roll(x, -1, axis=ax)
    t /= 7.0
    mask = np.zeros_like(t)
    mask[:, 2:-2, 2:-2, 2:-2] = 1.0
    net = fac.CNN(max_batch=n, seed=5)
    xd, td, md = (torch.from_numpy(a).cuda() for a in (x, t, mask))
    losses = [net.train_step(xd.data_ptr(), td.data_ptr(), md.data_ptr(), n, mask.sum(), 3e-3)
              for _ in range(150)]
    assert losses[-1] < 0.3 * losses[0], (losses[0], losses[-1])
    net.close()


def test_batch_walk_matches_single_samples(require_gpu):
    """A batch of many samples (each CTA of the tensor-core convolution walks
    several slabs, its accumulator barrier changing phase between them) gives
    bit for bit what the same samples give alone."""
    import torch
    rng = np.random.default_rng(2)
    n = 160
    net = fac.CNN(max_batch=n, seed=7)
    x = torch.from_numpy(rng.standard_normal((n, S, S, S)).astype(np.float32)).cuda()
    y = torch.zeros_like(x)
    net.forward(x.data_ptr(), n, y.data_ptr())
    for first in (0, 77, n - 2):
        xs = x[first:first + 2].contiguous()
        ys = torch.zeros_like(xs)
        net.forward(xs.data_ptr(), 2, ys.data_ptr())
        assert torch.equal(ys, y[first:first + 2])
    assert torch.isfinite(y).all()
    net.close()
