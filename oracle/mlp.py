"""CPU restatement of the learned warm-start network (test infrastructure).

Checks the CUDA kernels of urban-sph_a100_b200/csrc/learned.cu: the FP32
training forward/backward (gradients in FP64 here) and the tensor-core
inference, whose BF16 rounding of the weights and of the first hidden layer is
reproduced bit for bit before the FP32 sums.  Parameter layout (5569 floats):
W1[20][64], b1[64], W2[64][64], b2[64], w3[64], b3.
"""
import numpy as np

F, H = 20, 64
OW1, OB1 = 0, F * H
OW2 = OB1 + H
OB2 = OW2 + H * H
OW3 = OB2 + H
OB3 = OW3 + H
NPARAM = OB3 + 1


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[OW1:OB1].reshape(F, H), w[OB1:OW2], w[OW2:OB2].reshape(H, H), w[OB2:OW3], w[OW3:OB3], w[OB3])


def bf16_bits_to_float(bits):
    return (np.asarray(bits, np.uint32) << 16).view(np.float32)


def round_bf16(x):
    """Round-to-nearest-even of float32 values to BF16, returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return bf16_bits_to_float(u.astype(np.uint32))


def forward(w, X):
    """FP64 forward; X: rows x 20 (or 32) features."""
    W1, b1, W2, b2, w3, b3 = unpack(w)
    X = np.asarray(X, np.float64)[:, :F]
    h1 = np.maximum(X @ W1 + b1, 0)
    h2 = np.maximum(h1 @ W2 + b2, 0)
    return h2 @ w3 + b3, (X, h1, h2)


def loss_and_grad(w, X, t):
    """Mean squared error over the rows and its gradient (FP64)."""
    W1, b1, W2, b2, w3, b3 = unpack(w)
    y, (X, h1, h2) = forward(w, X)
    e = y - np.asarray(t, np.float64)
    n = len(e)
    dy = 2.0 * e / n
    g = np.zeros(NPARAM)
    g[OW3:OB3] = h2.T @ dy
    g[OB3] = dy.sum()
    d2 = np.outer(dy, w3) * (h2 > 0)
    g[OW2:OB2] = (h1.T @ d2).ravel()
    g[OB2:OW3] = d2.sum(0)
    d1 = (d2 @ W2.T) * (h1 > 0)
    g[OW1:OB1] = (X.T @ d1).ravel()
    g[OB1:OW2] = d1.sum(0)
    return float((e * e).mean()), g


def infer_bf16(w, X):
    """The tensor-core inference: BF16 weights and first hidden layer, FP32 sums."""
    W1, b1, W2, b2, w3, b3 = unpack(w)
    X = np.asarray(X, np.float32)[:, :F]
    W1r = round_bf16(W1.astype(np.float32)).astype(np.float64)
    W2r = round_bf16(W2.astype(np.float32)).astype(np.float64)
    h1 = np.maximum(X.astype(np.float64) @ W1r + b1.astype(np.float32), 0).astype(np.float32)
    h1r = round_bf16(h1).astype(np.float64)
    h2 = np.maximum(h1r @ W2r + b2.astype(np.float32), 0)
    return (h2 @ w3.astype(np.float32) + np.float32(b3)).astype(np.float32)
