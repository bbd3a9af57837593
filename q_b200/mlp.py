"""The lambda-placement network on the tensor cores (include/qb_mlp.h).

A 12 -> 64 -> 64 -> 11 perceptron with SiLU, whose forward pass, gradient and
Adam training run in hand-written tcgen05 kernels (BF16 operands, FP32
accumulation in tensor memory).  Parameters are one float32 vector in the
header's layout; `init` gives a He-style start.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib

IN, HID, OUT = 12, 64, 11
NPARAM = HID * IN + HID + HID * HID + HID + OUT * HID + OUT
MAX_SAMPLES = 4096


class Adam(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("weight_decay", C.c_float)]


def _f32(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if shape is not None and a.shape != shape:
        raise ValueError("expected shape %s, got %s" % (shape, a.shape))
    return a


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def init(seed: int = 0, zero_output: bool = False) -> np.ndarray:
    """He-style initial weights, biases zero; with zero_output the output
    layer starts at zero, so the untrained network outputs 0."""
    rng = np.random.default_rng(seed)
    w3 = rng.normal(0, np.sqrt(1.0 / HID), (OUT, HID))
    parts = [rng.normal(0, np.sqrt(2.0 / IN), (HID, IN)), np.zeros(HID),
             rng.normal(0, np.sqrt(2.0 / HID), (HID, HID)), np.zeros(HID),
             np.zeros_like(w3) if zero_output else w3, np.zeros(OUT)]
    return np.concatenate([q.reshape(-1) for q in parts]).astype(np.float32)


def forward(params, x, device: int = 0) -> np.ndarray:
    p = _f32(params, (NPARAM,))
    x = _f32(x)
    n = x.shape[0]
    y = np.zeros((n, OUT), dtype=np.float32)
    check(lib.qb_mlp_forward(_p(p), _p(x), n, _p(y), device))
    return y


def loss_grad(params, x, t, device: int = 0) -> tuple[float, np.ndarray]:
    p = _f32(params, (NPARAM,))
    x, t = _f32(x), _f32(t)
    L = np.zeros(1, dtype=np.float32)
    g = np.zeros(NPARAM, dtype=np.float32)
    check(lib.qb_mlp_loss_grad(_p(p), _p(x), _p(t), x.shape[0], _p(L), _p(g), device))
    return float(L[0]), g


def train(params, x, t, iters: int, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999,
          eps: float = 1e-8, weight_decay: float = 0.0, device: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Full-batch Adam (decoupled weight decay on the weight matrices) on the
    mean squared error; returns the trained parameters and the loss before
    every step."""
    p = _f32(params, (NPARAM,)).copy()
    x, t = _f32(x), _f32(t)
    hist = np.zeros(iters, dtype=np.float32)
    a = Adam(lr, beta1, beta2, eps, weight_decay)
    check(lib.qb_mlp_train(_p(p), _p(x), _p(t), x.shape[0], iters, C.addressof(a), _p(hist), device))
    return p, hist
