"""ORACLE (test infrastructure only): FP64 numpy restatement of the learned
eddy-viscosity closure -- features, training targets from box-filtered fields, the
6-32-32-1 MLP forward pass and its backward pass.

The closure has no counterpart in the reference (its eddy viscosity is the fixed
Smagorinsky term of lbm.cu:42-60, restated in oracle.cpp); this module pins the
engine's closure kernels against the mathematics they implement:
  * features / targets  -> lbl_closure_generate's filter and sample kernels
  * forward             -> the stream-collide's tensor-core inference and the
                           per-thread form (lbl_closure_infer), under the engine's
                           operand contract (BF16 parameters, FP16 matrix operands)
  * loss_and_grad       -> the fused forward/backward training kernel
The gradient itself is pinned against central finite differences in FP64.
Only tests/ use this module.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID = 6, 32
W1, B1 = 0, N_HID * N_IN
W2 = B1 + N_HID
B2 = W2 + N_HID * N_HID
W3 = B2 + N_HID
B3 = W3 + N_HID
N_PARAMS = B3 + 1  # 1313

GELU_K, GELU_C = 0.7978845608028654, 0.044715


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def f16(x) -> np.ndarray:
    """Round to the nearest FP16 (ties to even), returned as float64."""
    return np.asarray(x, dtype=np.float64).astype(np.float16).astype(np.float64)


def contract_params(params) -> np.ndarray:
    """Parameters as the engine uses them: BF16 values, the matrix operands W1, b1
    (the weight of a constant input), W2 and W3 carried in FP16."""
    p = bf16(params)
    p[W1:B2] = f16(p[W1:B2])
    p[W3:B3] = f16(p[W3:B3])
    return p


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[W1:B1].reshape(N_HID, N_IN), p[B1:W2], p[W2:B2].reshape(N_HID, N_HID), p[B2:W3], p[W3:B3], p[B3])


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(GELU_K * (x + GELU_C * x ** 3)))


def gelu_grad(x):
    t = np.tanh(GELU_K * (x + GELU_C * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_K * (1.0 + 3.0 * GELU_C * x * x)


def softplus(z):
    return np.where(z > 20.0, z, np.log1p(np.exp(np.minimum(z, 20.0))))


def sigmoid(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(params, x, contract: bool = True):
    """Multiplier m for feature rows x [n][6].  contract applies the engine's
    arithmetic contract: BF16 parameter values, FP16 matrix operands (weights,
    features, both hidden activations); everything else in FP64 here."""
    p = contract_params(params) if contract else np.asarray(params, np.float64)
    w1, b1, w2, b2, w3, b3 = unpack(p)
    x = f16(x) if contract else np.asarray(x, np.float64)
    h1 = x @ w1.T + b1
    a1 = gelu(h1)
    a1q = f16(a1) if contract else a1
    h2 = a1q @ w2.T + b2
    a2 = gelu(h2)
    a2q = f16(a2) if contract else a2
    z = a2q @ w3 + b3
    return softplus(z), (x, h1, a1q, h2, a2q, z)


def loss_and_grad(params, x, t, contract: bool = True):
    """Mean-square loss over the rows and its gradient with respect to the
    parameters (the contract's roundings pass the gradient straight through)."""
    p = contract_params(params) if contract else np.asarray(params, np.float64)
    w1, b1, w2, b2, w3, b3 = unpack(p)
    m, (xq, h1, a1q, h2, a2, z) = forward(params, x, contract)
    n = len(t)
    err = m - np.asarray(t, np.float64)
    loss = float(np.mean(err * err))
    dz = 2.0 * err / n * sigmoid(z)
    g = np.zeros(N_PARAMS)
    g[W3:B3] = a2.T @ dz
    g[B3] = dz.sum()
    d2 = np.outer(dz, w3) * gelu_grad(h2)
    g[W2:B2] = (d2.T @ a1q).ravel()
    g[B2:W3] = d2.sum(0)
    d1 = (d2 @ w2) * gelu_grad(h1)
    g[W1:B1] = (d1.T @ xq).ravel()
    g[B1:W2] = d1.sum(0)
    return loss, g


def features(ux, uy, vx, vy, dx, nu_ref, dx_ref):
    """The six closure inputs from the velocity gradient (FP64); returns (x [n][6], |S|)."""
    ux, uy, vx, vy = (np.asarray(a, np.float64).ravel() for a in (ux, uy, vx, vy))
    s12 = 0.5 * (uy + vx)
    w12 = 0.5 * (uy - vx)
    ss = ux * ux + 2 * s12 * s12 + vy * vy
    ww = 2 * w12 * w12
    smag, wmag = np.sqrt(2 * ss), np.sqrt(2 * ww)
    k = dx * dx / nu_ref
    x = np.stack([np.log1p(k * smag), np.log1p(k * wmag), (ww - ss) / (ww + ss + 1e-30),
                  (ux + vy) / np.sqrt(ss + 1e-30), np.full_like(ux, dx / dx_ref), np.arcsinh(k * (vx - uy))], axis=1)
    return x, smag


def box_filter(a, f: int):
    """Mean over f x f blocks of a [ny][nx] field."""
    ny, nx = a.shape
    return np.asarray(a, np.float64).reshape(ny // f, f, nx // f, f).mean(axis=(1, 3))


def samples(u, v, f: int, h: float, cs: float, dx: float, nu_ref: float, dx_ref: float):
    """Features and target multipliers of one fine (u, v) field filtered f x f: the
    coarse velocity gradient by periodic central differences over spacing h, and
    m* = -(tau_d : S) / (2 S:S) / ((cs dx)^2 |S|) clipped to [0, 8] (1 where S = 0)."""
    u = np.asarray(u, np.float64)
    v = np.asarray(v, np.float64)
    ub, vb = box_filter(u, f), box_filter(v, f)
    t11 = box_filter(u * u, f) - ub * ub
    t12 = box_filter(u * v, f) - ub * vb
    t22 = box_filter(v * v, f) - vb * vb

    def ddx(a):
        return (np.roll(a, -1, axis=1) - np.roll(a, 1, axis=1)) / (2 * h)

    def ddy(a):
        return (np.roll(a, -1, axis=0) - np.roll(a, 1, axis=0)) / (2 * h)

    ux, uy, vx, vy = ddx(ub), ddy(ub), ddx(vb), ddy(vb)
    x, smag = features(ux, uy, vx, vy, dx, nu_ref, dx_ref)
    s11, s22, s12 = ux.ravel(), vy.ravel(), 0.5 * (uy + vx).ravel()
    tr = 0.5 * (t11 + t22).ravel()
    ss = s11 * s11 + 2 * s12 * s12 + s22 * s22
    tds = (t11.ravel() - tr) * s11 + 2 * t12.ravel() * s12 + (t22.ravel() - tr) * s22
    base = cs * cs * dx * dx * smag
    ok = (ss > 1e-12) & (base > 0)
    m = np.ones_like(ss)
    m[ok] = -tds[ok] / (2 * ss[ok]) / base[ok]
    return x, np.clip(m, 0.0, 8.0)


def init_params(seed: int = 0) -> np.ndarray:
    """A seeded start in the engine's layout (Xavier-uniform weights, zero hidden
    biases, small output weights, softplus(b3) = 1) -- for tests."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS)
    for off, shape in ((W1, (N_HID, N_IN)), (W2, (N_HID, N_HID)), (W3, (1, N_HID))):
        a = np.sqrt(6.0 / (shape[0] + shape[1]))
        p[off:off + shape[0] * shape[1]] = rng.uniform(-a, a, shape[0] * shape[1])
    p[W3:B3] *= 0.1
    p[B3] = np.log(np.expm1(1.0))
    return p.astype(np.float32)
