"""The CPU restatement of the coarse-correction CNN: its analytic gradients
agree with central finite differences (FP32, no BF16 rounding), and BF16
rounding is round-to-nearest-even."""
import numpy as np

from oracle import cnn_oracle as co


def test_bf16_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7 + 2 ** -9, -3.140625, 1e-40], np.float32)
    r = co.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # tie -> even
    assert r[2] == np.float32(1.0 + 2 ** -7)   # 2^-9 above a representable value
    assert r[3] == np.float32(-3.140625)


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    net = co.CNN.init(seed=1, width=4, rounding=False)
    x = rng.standard_normal((2, 6, 6, 6)).astype(np.float32)
    t = rng.standard_normal((2, 6, 6, 6)).astype(np.float32)
    mask = np.zeros_like(t)
    mask[:, 1:-1, 1:-1, 1:-1] = 1.0
    loss, grads = net.loss_and_grads(x, t, mask)
    for li, idx in [(0, (4, 2)), (1, (13, 1, 3)), (2, (0, 2, 2)), (3, (26, 1))]:
        w = net.w[li]
        h = 1e-3
        old = w[idx]
        w[idx] = old + h
        lp, _ = net.loss_and_grads(x, t, mask)
        w[idx] = old - h
        lm, _ = net.loss_and_grads(x, t, mask)
        w[idx] = old
        fd = (lp - lm) / (2 * h)
        assert abs(fd - grads[li][idx]) <= 2e-3 * max(1.0, abs(fd)), (li, fd, grads[li][idx])
