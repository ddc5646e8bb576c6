"""CPU ORACLE for the learned Newton-iterate MLP — test infrastructure.

numpy restatement of the network the device kernels implement
(fvmpor_b200/csrc/predictor.cu): 8 normalised inputs -> 3 hidden layers of
64 with exact (erf) GELU -> 1 output, BF16 weights and BF16 layer inputs,
FP32 accumulation, loss = mean((y_hat - y)^2).  The backward pass mirrors the
device's rounding points (dZ rounded to BF16 before the dZ W product and
the dW accumulation).  Used only by tests/ to check the tensor-core
forward and backward kernels.  The reference has no such network, so this
oracle is pinned by finite differences (tests/test_gpu_mlp.py).
"""
import math

import numpy as np

IN, H = 8, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H * H
OFF_W4 = OFF_B3 + H
OFF_B4 = OFF_W4 + H
N_TRAIN = OFF_B4 + 1
OFF_MU = N_TRAIN
OFF_SD = OFF_MU + IN
N_PARAM = OFF_SD + IN

_erf = np.vectorize(math.erf, otypes=[np.float64])


def bf16(x):
    """round-to-nearest-even to bfloat16, returned as float32"""
    x = np.asarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def gelu(x):
    return (0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))).astype(np.float32)


def gelu_grad(x):
    cdf = 0.5 * (1.0 + _erf(x / math.sqrt(2.0)))
    pdf = np.exp(-0.5 * x.astype(np.float64) ** 2) / math.sqrt(2.0 * math.pi)
    return (cdf + x * pdf).astype(np.float32)


def unpack(P):
    P = np.asarray(P)
    if P.dtype != np.float64:
        P = P.astype(np.float32)
    return dict(
        W1=P[OFF_W1:OFF_B1].reshape(H, IN), b1=P[OFF_B1:OFF_W2], W2=P[OFF_W2:OFF_B2].reshape(H, H),
        b2=P[OFF_B2:OFF_W3], W3=P[OFF_W3:OFF_B3].reshape(H, H), b3=P[OFF_B3:OFF_W4], w4=P[OFF_W4:OFF_B4],
        b4=P[OFF_B4], mu=P[OFF_MU:OFF_SD], sd=np.where(P[OFF_SD:N_PARAM] > 0, P[OFF_SD:N_PARAM], 1.0))


def init_params(seed=0, mu=None, sd=None):
    rng = np.random.default_rng(seed)
    P = np.zeros(N_PARAM, np.float32)
    P[OFF_W1:OFF_B1] = rng.normal(0, 1 / math.sqrt(IN), H * IN)
    P[OFF_W2:OFF_B2] = rng.normal(0, 1 / math.sqrt(H), H * H)
    P[OFF_W3:OFF_B3] = rng.normal(0, 1 / math.sqrt(H), H * H)
    P[OFF_W4:OFF_B4] = rng.normal(0, 1 / math.sqrt(H), H)
    P[OFF_MU:OFF_SD] = 0.0 if mu is None else mu
    P[OFF_SD:N_PARAM] = 1.0 if sd is None else sd
    return P


def _round(exact):
    return (lambda a: np.asarray(a, np.float64)) if exact else bf16


def forward(P, X, keep=False, exact=False):
    """exact=True drops the BF16 rounding and computes in FP64 (used to pin
    the backward formulas against finite differences)"""
    r = _round(exact)
    dt = np.float64 if exact else np.float32
    p = {k: np.asarray(v, dt) for k, v in unpack(P).items()}
    x = r((np.asarray(X, dt) - p["mu"]) / p["sd"])
    W1, W2, W3 = r(p["W1"]), r(p["W2"]), r(p["W3"])
    act = _gelu64 if exact else gelu
    z1 = x @ W1.T + p["b1"]
    a1 = r(act(z1))
    z2 = a1 @ W2.T + p["b2"]
    a2 = r(act(z2))
    z3 = a2 @ W3.T + p["b3"]
    h3 = act(z3)
    out = h3 @ p["w4"] + p["b4"]
    if keep:
        return out, dict(x=x, z1=z1, a1=a1, z2=z2, a2=a2, z3=z3, h3=h3, W2=W2, W3=W3, p=p)
    return out


def grad(P, X, Y, exact=False):
    """gradient of mean((out - y)^2) w.r.t. the trainable parameters, and the loss"""
    r = _round(exact)
    gg = (lambda z: _gelu_grad64(z)) if exact else gelu_grad
    out, c = forward(P, X, keep=True, exact=exact)
    p = c["p"]
    n = len(Y)
    e = out - np.asarray(Y, out.dtype)
    dout = 2.0 * e / n
    g = np.zeros(N_TRAIN, np.float64 if exact else np.float32)
    g[OFF_W4:OFF_B4] = c["h3"].T @ dout
    g[OFF_B4] = dout.sum()
    dz3 = np.outer(dout, p["w4"]) * gg(c["z3"])
    dz3b = r(dz3)
    g[OFF_B3:OFF_W4] = dz3.sum(0)
    g[OFF_W3:OFF_B3] = (dz3b.T @ c["a2"]).ravel()
    da2 = dz3b @ c["W3"]
    dz2 = da2 * gg(c["z2"])
    dz2b = r(dz2)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    g[OFF_W2:OFF_B2] = (dz2b.T @ c["a1"]).ravel()
    da1 = dz2b @ c["W2"]
    dz1 = da1 * gg(c["z1"])
    dz1b = r(dz1)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_W1:OFF_B1] = (dz1b.T @ c["x"]).ravel()
    return g, float(np.mean(np.asarray(e, np.float64) ** 2))


def _gelu64(x):
    x = np.asarray(x, np.float64)
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def _gelu_grad64(x):
    x = np.asarray(x, np.float64)
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)
