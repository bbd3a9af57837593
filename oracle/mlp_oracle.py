"""CPU oracle of the lambda-placement network (test infrastructure only).

A numpy FP64 restatement of the 12 -> 64 -> 64 -> 11 SiLU perceptron of
q_b200/csrc/mlp.cu: forward pass, mean-squared-error loss, gradient of every
parameter, and Adam.  With bf16=True the operands are rounded to BF16 (round to
nearest even) at the points where the tensor-core kernel rounds them -- the
input, the weights, both hidden activations and the three pre-activation
gradients -- and everything else stays FP64, so the kernel's FP32 accumulation
is the remaining difference.  The network has no counterpart in the reference:
parity is against this restatement and against finite differences of it.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 12, 64, 11
SHAPES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (OUT, HID)), ("b3", (OUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    out, k = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[k:k + n], dtype=np.float64).reshape(shape)
        k += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).reshape(-1) for name, _ in SHAPES])


def bf16(a):
    """Round to the nearest BF16 value (ties to even), via float32."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x, bf=False):
    W = unpack(p)
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    x = r(x)
    z1 = x @ r(W["W1"]).T + W["b1"]
    h1 = r(_silu(z1))
    z2 = h1 @ r(W["W2"]).T + W["b2"]
    h2 = r(_silu(z2))
    y = h2 @ r(W["W3"]).T + W["b3"]
    return y, (x, z1, h1, z2, h2)


def loss_grad(p, x, t, bf=False):
    """Mean squared error over all n x 11 outputs and its gradient."""
    W = unpack(p)
    r = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    y, (xr, z1, h1, z2, h2) = forward(p, x, bf)
    n = len(x)
    e = y - t
    L = float(np.mean(e * e))
    d3 = 2.0 * e / (n * OUT)
    g = {"b3": d3.sum(0), "W3": r(d3).T @ h2}
    dh2 = r(d3) @ r(W["W3"])
    d2 = dh2 * _dsilu(z2)
    g["b2"] = d2.sum(0)
    g["W2"] = r(d2).T @ h1
    dh1 = r(d2) @ r(W["W2"])
    d1 = dh1 * _dsilu(z1)
    g["b1"] = d1.sum(0)
    g["W1"] = r(d1).T @ xr
    return L, pack(g)


def weight_mask():
    """1 for the entries of the weight matrices, 0 for the biases."""
    return pack({name: np.ones(shape) if name.startswith("W") else np.zeros(shape) for name, shape in SHAPES})


def train(p, x, t, iters, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0, bf=False):
    """Full-batch Adam with decoupled weight decay on the weight matrices;
    returns the parameters and the loss before each step."""
    p = np.array(p, dtype=np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    wd = weight_decay * weight_mask()
    losses = []
    for it in range(1, iters + 1):
        L, g = loss_grad(p, x, t, bf)
        losses.append(L)
        m = beta1 * m + (1 - beta1) * g
        v = beta2 * v + (1 - beta2) * g * g
        p -= lr * ((m / (1 - beta1 ** it)) / (np.sqrt(v / (1 - beta2 ** it)) + eps) + wd * p)
    return p, np.array(losses)


def init(seed=0):
    """He-style initialisation, biases zero."""
    rng = np.random.default_rng(seed)
    d = {"W1": rng.normal(0, np.sqrt(2.0 / IN), (HID, IN)), "b1": np.zeros(HID),
         "W2": rng.normal(0, np.sqrt(2.0 / HID), (HID, HID)), "b2": np.zeros(HID),
         "W3": rng.normal(0, np.sqrt(1.0 / HID), (OUT, HID)), "b3": np.zeros(OUT)}
    return pack(d)
