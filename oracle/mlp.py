"""CPU oracle of the learned cardinality estimator's network (test infrastructure only:
the tests import it to check the device kernels; nothing in the engine calls it).

The reference has no such component (it sizes buffers from the free device memory,
cm.cu:3184), so this restates the network the engine defines: 64 -> 128 -> 128 -> 3 with
ReLU, weights rounded to BF16 (round to nearest even) for the forward and backward passes,
accumulation in float64 here (the device accumulates in FP32), masked mean squared error,
and Adam on FP32 master weights. Parameters are flat, in the order W1[128][64], b1[128],
W2[128][128], b2[128], W3[3][128], b3[3].
"""
import numpy as np

N_IN, N_HID, N_OUT = 64, 128, 3
SHAPES = [(N_HID, N_IN), (N_HID,), (N_HID, N_HID), (N_HID,), (N_OUT, N_HID), (N_OUT,)]
N_PARAMS = sum(int(np.prod(s)) for s in SHAPES)


def bf16_round(a):
    """float32 values rounded to the nearest BF16 value (ties to even), as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16 << 16
    return u.astype(np.uint32).view(np.float32)


def bf16_bits_to_f32(bits):
    return (np.asarray(bits, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def unpack(p):
    out, o = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        out.append(np.asarray(p[o:o + n]).reshape(s))
        o += n
    return out


def forward(p, x, bf16=True):
    """Outputs and the activations the backward pass needs (weights BF16-rounded)."""
    if bf16:  # FP32 master parameters, BF16 weights
        W1, b1, W2, b2, W3, b3 = unpack(np.asarray(p, dtype=np.float32))
        W1, W2, W3 = bf16_round(W1), bf16_round(W2), bf16_round(W3)
    else:  # the parameters as given, in float64
        W1, b1, W2, b2, W3, b3 = unpack(np.asarray(p, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = (a.astype(np.float64) for a in (W1, b1, W2, b2, W3, b3))
    x = np.asarray(x, dtype=np.float64)
    h1 = np.maximum(x @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    y = h2 @ W3.T + b3
    return y, (x, h1, h2, W1, W2, W3)


def loss_and_grad(p, x, t, mask, bf16=True):
    """Masked MSE sum((y - t)^2 * mask) / n and its gradient (flat, parameter order)."""
    y, (x, h1, h2, W1, W2, W3) = forward(p, x, bf16)
    n = x.shape[0]
    e = (y - t) * mask
    loss = float((e * e).sum() / n)
    dy = 2.0 * e / n
    gW3, gb3 = dy.T @ h2, dy.sum(0)
    d2 = (dy @ W3) * (h2 > 0)
    gW2, gb2 = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ W2) * (h1 > 0)
    gW1, gb1 = d1.T @ x, d1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss, g


def adam_step(p, g, m1, m2, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update (step counts from 1); returns new (p, m1, m2)."""
    m1 = b1 * m1 + (1 - b1) * g
    m2 = b2 * m2 + (1 - b2) * g * g
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    p = p - lr * (m1 / c1) / (np.sqrt(m2 / c2) + eps)
    return p, m1, m2
