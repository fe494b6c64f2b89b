"""CPU restatement (float64 numpy) of the selector MLP's forward and backward
passes -- test infrastructure: the checker for the engine's training kernels
(kratos_b200/csrc/kr_learn.cu, k_mlp_grad) and its BF16 inference path.

Network: 16 -> 32 (ReLU) -> 32 (ReLU) -> 1 logit.  Parameters in one flat
vector: W1[16][32], b1[32], W2[32][32], b2[32], W3[32], b3 (row-major [in][out]).
Loss: class-weighted binary cross-entropy on the logit, weight 1 for y = 1 and
wneg for y = 0, averaged over samples.
"""
import numpy as np

N_IN, N_H = 16, 32
OFF = {}
_o = 0
for _name, _n in (("W1", N_IN * N_H), ("b1", N_H), ("W2", N_H * N_H), ("b2", N_H), ("W3", N_H), ("b3", 1)):
    OFF[_name] = (_o, _o + _n)
    _o += _n
N_PARAM = _o


def unpack(w):
    w = np.asarray(w, np.float64)
    g = lambda k: w[OFF[k][0]:OFF[k][1]]
    return g("W1").reshape(N_IN, N_H), g("b1"), g("W2").reshape(N_H, N_H), g("b2"), g("W3"), g("b3")[0]


def forward(X, w):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    X = np.asarray(X, np.float64)
    a1 = X @ W1 + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2 + b2
    h2 = np.maximum(a2, 0)
    z = h2 @ W3 + b3
    return z, (X, h1, h2)


def loss_grad(X, y, w, wneg=1.0):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    z, (X, h1, h2) = forward(X, w)
    y = np.asarray(y, np.float64)
    wy = np.where(y > 0.5, 1.0, wneg)
    n = len(y)
    loss = (wy * (np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))).sum() / n
    dz = wy * (1 / (1 + np.exp(-z)) - y)
    d2 = (dz[:, None] * W3[None, :]) * (h2 > 0)
    d1 = (d2 @ W2.T) * (h1 > 0)
    g = np.concatenate([(X.T @ d1).ravel(), d1.sum(0), (h1.T @ d2).ravel(), d2.sum(0),
                        h2.T @ dz, [dz.sum()]]) / n
    return loss, g


def bf16(x):
    """Round float32 values to bfloat16 (round to nearest even), as float32."""
    a = np.asarray(x, np.float32).copy()
    u = a.view(np.uint32)
    u += 0x7FFF + ((u >> 16) & 1)
    u &= 0xFFFF0000
    return a


def forward_bf16(X, w):
    """Logits with the BF16 tensor-core path's roundings: inputs, weights and
    hidden activations rounded to bf16, sums in float64 (stand-in for FP32
    accumulate), biases in FP32."""
    W1, b1, W2, b2, W3, b3 = unpack(w)
    Xb = bf16(X).astype(np.float64)
    h1 = bf16(np.maximum(Xb @ bf16(W1).astype(np.float64) + b1.astype(np.float32), 0)).astype(np.float64)
    h2 = bf16(np.maximum(h1 @ bf16(W2).astype(np.float64) + b2.astype(np.float32), 0)).astype(np.float64)
    return h2 @ bf16(W3).astype(np.float64) + np.float32(b3)
