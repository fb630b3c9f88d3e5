"""CPU oracle of the rank-predictor MLP (test infrastructure only).

Restates dense_hodlr_b200/csrc/rank_mlp.cu in NumPy, to check the CUDA
forward pass and gradients: 14 -> 64 -> 64 -> 1 with GELU, inputs
standardised and every input, weight and hidden activation rounded to BF16
at the same points as the CUDA kernels (round to nearest even).  The
forward pass is float32 in the kernels' summation order (bit for bit up to
erf's last bit); the backward pass is float64.  Loss 1/B sum (y - t)^2.
The reference has no learned part; this is the oracle of the project's own
predictor.

With bf16_round=False nothing is rounded and all arithmetic is float64, so
the gradient can be checked against central finite differences.
"""
import math

import numpy as np

NI, NH = 14, 64
OFF_MEAN, OFF_ISTD = 0, NI
OFF_W1 = 2 * NI
OFF_B1 = OFF_W1 + NH * NI
OFF_W2 = OFF_B1 + NH
OFF_B2 = OFF_W2 + NH * NH
OFF_W3 = OFF_B2 + NH
OFF_B3 = OFF_W3 + NH
NPARAM = OFF_B3 + 1
NTRAIN = NPARAM - 2 * NI


def bf16(x):
    """Round float32 values to BF16 (nearest even); returns float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf)


def gelu(a):
    return 0.5 * a * (1.0 + _erf(a / math.sqrt(2.0)))


def gelu_d(a):
    return 0.5 * (1.0 + _erf(a / math.sqrt(2.0))) + a * np.exp(-0.5 * a * a) / math.sqrt(2 * math.pi)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return dict(mean=p[OFF_MEAN:OFF_MEAN + NI], istd=p[OFF_ISTD:OFF_ISTD + NI],
                W1=p[OFF_W1:OFF_B1].reshape(NH, NI), b1=p[OFF_B1:OFF_W2],
                W2=p[OFF_W2:OFF_B2].reshape(NH, NH), b2=p[OFF_B2:OFF_W3],
                W3=p[OFF_W3:OFF_B3], b3=p[OFF_B3])


def _gelu32(a):
    """GELU in float32 operations as the kernel writes it,
    0.5f * a * (1 + erf(a * 0.70710678f)) (erf correctly rounded here)."""
    f = np.float32
    t = (a * f(0.70710678)).astype(f)
    e = _erf(t.astype(np.float64)).astype(f)
    return ((f(0.5) * a).astype(f) * (f(1.0) + e).astype(f)).astype(f)


def _dense32(b, W, h):
    """b + W h per sample, accumulated in float32 in input order.  Products of
    BF16 values are exact in float32, so each step rounds once, as fmaf."""
    f = np.float32
    a = np.broadcast_to(np.asarray(b, f), (h.shape[0], W.shape[0])).copy()
    for i in range(W.shape[1]):
        a = (a + (W[:, i].astype(f)[None, :] * h[:, i].astype(f)[:, None])).astype(f)
    return a


def forward(p, X, bf16_round=True):
    """y and the activations of a batch X (B x 14).  With BF16 rounding the
    arithmetic is float32 in the kernel's order; otherwise float64."""
    q = unpack(p)
    if bf16_round:
        f = np.float32
        x = bf16((np.asarray(X, f) - q["mean"].astype(f)) * q["istd"].astype(f))
        W1, W2, W3 = bf16(q["W1"]), bf16(q["W2"]), bf16(q["W3"])
        a1 = _dense32(q["b1"], W1, x)
        h1 = bf16(_gelu32(a1))
        a2 = _dense32(q["b2"], W2, h1)
        h2 = bf16(_gelu32(a2))
        y = _dense32(np.array([q["b3"]]), W3[None, :], h2)[:, 0].astype(np.float64)
        a1, a2 = a1.astype(np.float64), a2.astype(np.float64)
    else:
        x = (np.asarray(X, np.float64) - q["mean"]) * q["istd"]
        W1, W2, W3 = q["W1"], q["W2"], q["W3"]
        a1 = x @ W1.T + q["b1"]
        h1 = gelu(a1)
        a2 = h1 @ W2.T + q["b2"]
        h2 = gelu(a2)
        y = h2 @ W3 + q["b3"]
    return y, dict(x=x, a1=a1, h1=h1, a2=a2, h2=h2, W2=W2, W3=W3)


def loss_grad(p, X, T, bf16_round=True):
    """Loss and gradient of the trained parameters (blob order after the
    standardisation block), as mlp_sample_kernel + mlp_param_kernel."""
    y, c = forward(p, X, bf16_round)
    B = len(y)
    e = y - np.asarray(T, np.float64)
    dy = 2.0 * e / B
    da2 = dy[:, None] * c["W3"][None, :] * gelu_d(c["a2"])
    da1 = (da2 @ c["W2"]) * gelu_d(c["a1"])
    g = np.concatenate([(da1.T @ c["x"]).ravel(), da1.sum(0), (da2.T @ c["h1"]).ravel(),
                        da2.sum(0), dy @ c["h2"], [dy.sum()]])
    return float(np.mean(e * e)), g


def loss(p, X, T, bf16_round=True):
    y, _ = forward(p, X, bf16_round)
    return float(np.mean((y - np.asarray(T, np.float64)) ** 2))
