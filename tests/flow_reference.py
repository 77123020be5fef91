"""TEST INFRASTRUCTURE: the proposal network of pwa_b200.flow restated on the CPU with torch autograd in
float64 (or float32), as the checker of the GPU forward and backward kernels.

The network: input 2u - 1 in 7 of 64 columns (u = x, or the pre-maps' u = F(x)), four hidden layers
of 256 SiLU units, 8 x 64 output logits with autoregressive masks; log q(x) = sum_d [log 64 +
log softmax(logits_d)[floor(64 u_d)] + log F_d'(x_d)];
loss = -sum_i w_i log q(x_i) / sum_i w_i.  emulate_bf16 rounds what the GPU keeps in BF16 (weights,
the network input, the hidden activations) so that only the arithmetic precision differs."""
from __future__ import annotations

import numpy as np
import torch

D, BINS, IN = 7, 64, 64


def _bf16(t: torch.Tensor) -> torch.Tensor:
    return t.to(torch.bfloat16).to(t.dtype)


def premap_forward(cdf: np.ndarray, x: np.ndarray) -> tuple:
    """u = F(x) and log F'(x) of the piecewise-linear pre-maps (cdf [7, nodes]) at x [7, n]."""
    cells = cdf.shape[1] - 1
    k = np.clip(np.floor(x * cells).astype(np.int64), 0, cells - 1)
    t = x * cells - k
    a = np.take_along_axis(cdf, k, axis=1)
    b = np.take_along_axis(cdf, k + 1, axis=1)
    return a + t * (b - a), np.log((b - a) * cells).sum(axis=0)


def log_q(params, x: np.ndarray, dtype=torch.float64, emulate_bf16: bool = True, grad: bool = False, cdf=None):
    """log q of the events x [7, n] (numpy) and the parameter tensors (requires_grad when grad); cdf:
    the pre-maps' nodes (identity when None)."""
    n = x.shape[1]
    lpm = np.zeros(n)
    if cdf is not None:
        x, lpm = premap_forward(cdf, x)
    inp = torch.zeros((n, IN), dtype=dtype)
    inp[:, :D] = torch.as_tensor((2.0 * x - 1.0).T.astype(np.float32), dtype=dtype)
    if emulate_bf16:
        inp = _bf16(inp)
    ts = []
    h = inp
    for l, (W, b) in enumerate(params):
        Wt = torch.as_tensor(W, dtype=dtype)
        if emulate_bf16:
            Wt = _bf16(Wt)
        Wt.requires_grad_(grad)
        bt = torch.as_tensor(b, dtype=dtype).requires_grad_(grad)
        ts.append((Wt, bt))
        z = h @ Wt.T + bt
        if l < len(params) - 1:
            h = torch.nn.functional.silu(z)
            if emulate_bf16:
                h = h + (_bf16(h) - h).detach()  # rounded value, exact derivative
        else:
            h = z
    logits = h
    bins = torch.as_tensor(np.clip(np.floor(x * BINS), 0, BINS - 1).astype(np.int64).T)
    lq = torch.as_tensor(lpm, dtype=dtype)
    for d in range(D):
        lp = torch.log_softmax(logits[:, d * BINS:(d + 1) * BINS], dim=1)
        lq = lq + np.log(BINS) + lp.gather(1, bins[:, d:d + 1]).squeeze(1)
    return lq, ts


def loss_and_grads(params, x: np.ndarray, w: np.ndarray, emulate_bf16: bool = True):
    """(loss, [(dW, db)]) in float64 with autograd."""
    lq, ts = log_q(params, x, torch.float64, emulate_bf16, grad=True)
    wt = torch.as_tensor(w, dtype=torch.float64)
    loss = -(wt * lq).sum() / wt.sum()
    loss.backward()
    return float(loss.detach()), [(W.grad.numpy(), b.grad.numpy()) for W, b in ts]
