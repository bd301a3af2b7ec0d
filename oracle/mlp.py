"""CPU oracle for the learned initialiser's MLP -- TEST INFRASTRUCTURE ONLY.

The MLP (d -> 512 -> 512 -> dim, ReLU, mean-squared error, AdamW) has no counterpart in
beamform/pacmap-rs; it is the learned pattern added around the reference's Initialization::Value
(src/lib.rs:753-766), which rescales whatever the network predicts to std 1e-4. The GPU engine runs
it with BF16 weights and activations and FP32 accumulation; this module restates the same network in
numpy with the same rounding points (every GEMM operand rounded to BF16, round-to-nearest-even; sums in
float64) so the GPU gradients can be compared tensor by tensor. With ``bf16=False`` it is the plain
float64 network, which ``finite_difference`` checks against central differences -- the oracle's own
pin (there are no reference golden vectors for a component the reference does not have).

Only ``tests/`` import this module.
"""
from __future__ import annotations

import numpy as np

H = 512


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    if nan.any():
        out = out.copy()
        out[nan] = np.nan
    return out


def param_count(d: int, dim: int) -> int:
    return H * d + H + H * H + H + dim * H + dim


def unflatten(p: np.ndarray, d: int, dim: int):
    """Flat layout [W1 (512 x d), b1, W2 (512 x 512), b2, W3 (dim x 512), b3] -> tensors (views)."""
    p = np.asarray(p)
    o = 0
    out = []
    for shape in ((H, d), (H,), (H, H), (H,), (dim, H), (dim,)):
        cnt = int(np.prod(shape))
        out.append(p[o:o + cnt].reshape(shape))
        o += cnt
    assert o == p.size
    return out


def flatten(ts) -> np.ndarray:
    return np.concatenate([np.asarray(t, np.float64).ravel() for t in ts])


def _r(a, on):
    return bf16(a).astype(np.float64) if on else np.asarray(a, np.float64)


def forward(p, x, d: int, dim: int, bf16_ops: bool = True):
    """(Z1, H1, Z2, H2, out) for rows x (n x d); H1/H2 are the stored (BF16 when bf16_ops) activations."""
    W1, b1, W2, b2, W3, b3 = unflatten(p, d, dim)
    X = _r(x, bf16_ops)
    Z1 = X @ _r(W1, bf16_ops).T + b1
    H1 = _r(np.maximum(Z1, 0.0).astype(np.float32) if bf16_ops else np.maximum(Z1, 0.0), bf16_ops)
    Z2 = H1 @ _r(W2, bf16_ops).T + b2
    H2 = _r(np.maximum(Z2, 0.0).astype(np.float32) if bf16_ops else np.maximum(Z2, 0.0), bf16_ops)
    out = H2 @ _r(W3, bf16_ops).T + b3
    return Z1, H1, Z2, H2, out


def apply(p, x, d: int, dim: int, bf16_ops: bool = True) -> np.ndarray:
    return forward(p, x, d, dim, bf16_ops)[-1]


def loss_and_grad(p, x, t, d: int, dim: int, bf16_ops: bool = True):
    """Mean-squared error over the batch and its gradient in the flat layout.

    Rounding points of the GPU engine: dZ3 = 2 (out - t) / (B dim) -> BF16; dZ2 = (dZ3 . W3) * [H2 > 0]
    -> BF16; dZ1 = (dZ2 . W2) * [H1 > 0] -> BF16; weight gradients are FP32 sums of BF16 products; bias
    gradients are column sums of the BF16 dZ.
    """
    W1, b1, W2, b2, W3, b3 = unflatten(p, d, dim)
    B = x.shape[0]
    X = _r(x, bf16_ops)
    _, H1, _, H2, out = forward(p, x, d, dim, bf16_ops)
    e = out.astype(np.float32) - np.asarray(t, np.float32) if bf16_ops else out - np.asarray(t, np.float64)
    loss = float(np.sum(np.asarray(e, np.float64) ** 2) / (B * dim))
    scale = np.float32(2.0) / np.float32(B * dim)
    dZ3 = _r((np.float32(scale) * e).astype(np.float32) if bf16_ops else 2.0 * e / (B * dim), bf16_ops)
    gW3 = dZ3.T @ H2
    gb3 = dZ3.sum(0)
    dZ2 = dZ3 @ _r(W3, bf16_ops) * (H2 > 0)
    dZ2 = _r(dZ2.astype(np.float32) if bf16_ops else dZ2, bf16_ops)
    gW2 = dZ2.T @ H1
    gb2 = dZ2.sum(0)
    dZ1 = dZ2 @ _r(W2, bf16_ops) * (H1 > 0)
    dZ1 = _r(dZ1.astype(np.float32) if bf16_ops else dZ1, bf16_ops)
    gW1 = dZ1.T @ X
    gb1 = dZ1.sum(0)
    return loss, flatten([gW1, gb1, gW2, gb2, gW3, gb3])


def finite_difference(p, x, t, d: int, dim: int, idx, h: float = 1e-6) -> np.ndarray:
    """Central differences of the float64 loss at the flat parameter indices ``idx``."""
    p = np.asarray(p, np.float64).copy()
    out = []
    for i in idx:
        old = p[i]
        p[i] = old + h
        lp, _ = loss_and_grad(p, x, t, d, dim, bf16_ops=False)
        p[i] = old - h
        lm, _ = loss_and_grad(p, x, t, d, dim, bf16_ops=False)
        p[i] = old
        out.append((lp - lm) / (2 * h))
    return np.array(out)


def adamw(p, g, m, v, step: int, lr: float, wd: float, d: int, dim: int):
    """One AdamW step (beta 0.9 / 0.999, eps 1e-8; decoupled decay on the weight matrices only)."""
    decay = np.concatenate([np.full(s.size, wd if s.ndim == 2 else 0.0) for s in unflatten(p, d, dim)])
    m = 0.9 * m + 0.1 * g
    v = 0.999 * v + 0.001 * g * g
    mh = m / (1 - 0.9 ** step)
    vh = v / (1 - 0.999 ** step)
    p = p * (1 - lr * decay) - lr * mh / (np.sqrt(vh) + 1e-8)
    return p, m, v
