"""FP64 numpy oracle of the volume-move surrogate MLP (test infrastructure).

Same network as lcmc_mlp.cu: n_in -> 128 -> 128 -> 1 with SiLU, BF16 rounding
at the same points as the GPU (inputs, weights of the two matrix layers, first
hidden activations), everything else in FP64.  Gradients of the batch MSE by
hand-written backpropagation.
"""
import numpy as np


def bf16(x):
    """Round float32 values to BF16 (round to nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, n_in, hid=128):
    k1 = (n_in + 127) // 128 * 128
    o = 0
    W1 = params[o:o + hid * k1].reshape(hid, k1)[:, :n_in].astype(np.float64); o += hid * k1
    b1 = params[o:o + hid].astype(np.float64); o += hid
    W2 = params[o:o + hid * hid].reshape(hid, hid).astype(np.float64); o += hid * hid
    b2 = params[o:o + hid].astype(np.float64); o += hid
    w3 = params[o:o + hid].astype(np.float64); o += hid
    b3 = params[o:o + 1].astype(np.float64)
    return W1, b1, W2, b2, w3, b3, k1


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, x, n_in):
    W1, b1, W2, b2, w3, b3, _ = unpack(params, n_in)
    X = bf16(x)
    Z1 = X @ bf16(W1).T + b1
    H1 = bf16(silu(Z1))
    Z2 = H1 @ bf16(W2).T + b2
    A2 = silu(Z2)
    y = A2 @ w3 + b3[0]
    return y, (X, Z1, H1, Z2, A2)


def gradients(params, x, t, n_in):
    W1, b1, W2, b2, w3, b3, k1 = unpack(params, n_in)
    y, (X, Z1, H1, Z2, A2) = forward(params, x, n_in)
    n = len(t)
    e = y - t
    loss = float(np.mean(e * e))
    dy = 2.0 * e / n
    gw3 = A2.T @ dy
    gb3 = np.array([dy.sum()])
    dZ2 = np.outer(dy, w3) * dsilu(Z2)
    gW2 = dZ2.T @ H1
    gb2 = dZ2.sum(axis=0)
    dH1 = dZ2 @ W2
    dZ1 = dH1 * dsilu(Z1)
    gW1 = np.zeros((128, k1))
    gW1[:, :n_in] = dZ1.T @ X
    gb1 = dZ1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, gb3])
    return g, loss
