"""Training and evaluation of the learned coarse correction.

The network (fac_cnn_* kernels, BF16 convolutions on the tensor cores)
maps the composite residual on one patch plus a one-cell halo, scaled by
the patch's RMS residual, to the error on the patch interior in units of
that RMS times dx^2 (the convention of fac_set_learned).  Training pairs
come from the FAC solver itself: for a problem with converged solution u*,
the solver is restarted and stopped after k cycles; the residual r_k of
that state and the error e_k = u* - u_k on every patch of the learned level
form one pair per patch.  Training runs on the GPU with the project's own
forward / backward / Adam kernels (fac_cnn_train_step).  In the solver the
prediction is applied as a minimal-residual step per problem whose step
length is 0 whenever it would not lower the residual, so plain FAC is both
the fallback and the judge of the correction.
"""
from __future__ import annotations

import dataclasses
from typing import List, Sequence

import numpy as np

from . import configs, fac

S = fac.CNN_BOX
S3 = S * S * S


def level_dx(prob, ln):
    """Grid spacing along x of level ln."""
    n = prob.n0[0]
    for l in range(1, ln + 1):
        n *= prob.levels[l].ratio[0]
    return (prob.xup[0] - prob.xlo[0]) / n


@dataclasses.dataclass
class PairSet:
    """Training pairs on the device: inputs x, targets t and masks m, each
    of shape (n, S, S, S) FP32 torch tensors."""
    x: object
    t: object
    m: object

    @property
    def n(self):
        return int(self.x.shape[0])

    def cat(self, other):
        import torch
        return PairSet(torch.cat([self.x, other.x]), torch.cat([self.t, other.t]),
                       torch.cat([self.m, other.m]))


def _targets(prob, ln, err, scale, offset):
    """Host targets and masks for the patches of one problem: the error
    interior placed at offset 1 of each S^3 box (as the samples place the
    patch interior), divided by scale * dx^2."""
    dx2 = level_dx(prob, ln) ** 2
    boxes = prob.levels[ln].boxes
    t = np.zeros((len(boxes), S, S, S), dtype=np.float32)
    m = np.zeros((len(boxes), S, S, S), dtype=np.float32)
    for ip, (b, lo, v) in enumerate(configs.patch_views(prob, ln, err, 1)):
        nz, ny, nx = v.shape[0] - 2, v.shape[1] - 2, v.shape[2] - 2
        sc = scale[offset + ip]
        if not sc > 0:
            continue
        t[ip, 1:nz + 1, 1:ny + 1, 1:nx + 1] = v[1:-1, 1:-1, 1:-1] / (sc * dx2)
        m[ip, 1:nz + 1, 1:ny + 1, 1:nx + 1] = 1.0
    return t, m


def generate_pairs(problems: Sequence, level: int, cycles: Sequence[int], params=None,
                   precision="mixed", device=0) -> PairSet:
    """Pairs from FAC runs on `problems` (one context, solved together):
    for each k in `cycles`, the state after k cycles from a zero start."""
    import torch
    prm = dict(params or {})
    ctx = fac.FacContext(problems, params=prm, device=device, precision=precision)
    try:
        ctx.zero(fac.U)
        ctx.solve()
        ustar = [ctx.download(fac.U, i, level) for i in range(len(problems))]
        npatch = sum(len(p.levels[level].boxes) for p in problems)
        xs, ts, ms = [], [], []
        for k in cycles:
            ctx.set_params(max_cycles=int(k))
            ctx.zero(fac.U)
            ctx.solve()
            x = torch.empty((npatch, S, S, S), dtype=torch.float32, device=f"cuda:{device}")
            scale = ctx.learned_samples(level, x.data_ptr(), npatch)
            off = 0
            tt, mm = [], []
            for i, p in enumerate(problems):
                err = ustar[i] - ctx.download(fac.U, i, level)
                t, m = _targets(p, level, err, scale, off)
                tt.append(t)
                mm.append(m)
                off += len(p.levels[level].boxes)
            keep = torch.from_numpy(scale > 0)
            xs.append(x[keep.to(x.device)])
            ts.append(torch.from_numpy(np.concatenate(tt))[keep].to(x.device))
            ms.append(torch.from_numpy(np.concatenate(mm))[keep].to(x.device))
        return PairSet(torch.cat(xs), torch.cat(ts), torch.cat(ms))
    finally:
        ctx.close()


def masked_loss(net, pairs: PairSet, batch=256):
    """Mean masked squared error of the network on a pair set (no update)."""
    tot = 0.0
    cnt = 0.0
    for b in range(0, pairs.n, batch):
        e = min(pairs.n, b + batch)
        x, t, m = (a[b:e].contiguous() for a in (pairs.x, pairs.t, pairs.m))
        loss, _ = net.gradients(x.data_ptr(), t.data_ptr(), m.data_ptr(), e - b)
        ms = float(m.sum())
        tot += loss * ms
        cnt += ms
    return tot / max(cnt, 1.0)


def train(net, pairs: PairSet, epochs=4, batch=64, lr=1e-3, seed=0, log=None):
    """Adam on the masked MSE over shuffled mini-batches; returns the mean
    loss of each epoch."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    losses = []
    for ep in range(epochs):
        perm = torch.randperm(pairs.n, generator=g).to(pairs.x.device)
        tot, cnt = 0.0, 0
        for b in range(0, pairs.n - batch + 1, batch):
            idx = perm[b:b + batch]
            x, t, m = (a.index_select(0, idx).contiguous() for a in (pairs.x, pairs.t, pairs.m))
            ms = float(m.sum())
            if ms <= 0:
                continue
            loss = net.train_step(x.data_ptr(), t.data_ptr(), m.data_ptr(), batch, ms, lr)
            tot += loss
            cnt += 1
        losses.append(tot / max(cnt, 1))
        if log:
            log(f"epoch {ep}: loss {losses[-1]:.4e}")
    return losses


def evaluate(problems: Sequence, level: int, net, params=None, precision="mixed", device=0,
             krylov=0):
    """Solve `problems` without and with the learned correction; returns
    per-variant cycles, final residuals, residual histories and device ms.
    With krylov > 0 the solves are FGMRES(krylov), the network being the
    second stage of the preconditioner (after the FAC cycle); else the
    stationary FAC loop with the network's minimal-residual step after every
    cycle."""
    out = {}
    for name, use in (("plain", False), ("learned", True)):
        ctx = fac.FacContext(problems, params=dict(params or {}), device=device,
                             precision=precision)
        try:
            if krylov:
                ctx.set_krylov(krylov)
            if use:
                ctx.set_learned(net, level)
            ctx.zero(fac.U)
            ctx.solve()  # warm-up (graph capture)
            ctx.zero(fac.U)
            ctx.timer_start()
            conv, its, res = ctx.solve()
            ms = ctx.timer_stop()
            out[name] = dict(converged=conv.copy(), cycles=its.copy(), residual=res.copy(),
                             history=[ctx.residual_history(i) for i in range(len(problems))],
                             ms=ms)
        finally:
            ctx.close()
    return out


# FLOPs per sample cell of one training step (forward, data gradients of
# layers 4..2, weight gradients of all four layers; a multiply-add is two):
# forward 2*27*(1*16 + 16*16 + 16*16 + 16*1), data backward the same minus
# layer 1, weight gradients the same as forward.
FWD_FLOP_PER_CELL = 2 * 27 * (16 + 256 + 256 + 16)
TRAIN_FLOP_PER_CELL = 2 * FWD_FLOP_PER_CELL + 2 * 27 * (256 + 256 + 16)


def training_throughput(net, batch=256, steps=20, device=0, seed=0):
    """Training throughput of the project's kernels on random samples:
    TFLOP/s of fac_cnn_train_step (wall time of `steps` steps of `batch`
    samples between device synchronisations) and of the forward pass."""
    import time

    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    shape = (batch, S, S, S)
    x = torch.randn(shape, generator=g).to(f"cuda:{device}")
    t = torch.randn(shape, generator=g).to(f"cuda:{device}")
    m = torch.ones(shape, device=f"cuda:{device}")
    y = torch.empty(shape, device=f"cuda:{device}")
    ms = float(m.sum())
    for _ in range(3):
        net.train_step(x.data_ptr(), t.data_ptr(), m.data_ptr(), batch, ms, 1e-4)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(steps):
        net.train_step(x.data_ptr(), t.data_ptr(), m.data_ptr(), batch, ms, 1e-4)
    torch.cuda.synchronize(device)
    train_s = (time.perf_counter() - t0) / steps
    for _ in range(3):
        net.forward(x.data_ptr(), batch, y.data_ptr())
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    for _ in range(steps):
        net.forward(x.data_ptr(), batch, y.data_ptr())
    torch.cuda.synchronize(device)
    fwd_s = (time.perf_counter() - t0) / steps
    cells = batch * S3
    return {"batch": batch, "train_ms": train_s * 1e3, "forward_ms": fwd_s * 1e3,
            "train_tflops": cells * TRAIN_FLOP_PER_CELL / train_s / 1e12,
            "forward_tflops": cells * FWD_FLOP_PER_CELL / fwd_s / 1e12}
