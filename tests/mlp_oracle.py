"""numpy fp32 reference of the cost-model MLP forward/backward (test
infrastructure): bf16-rounded weights and activations, fp32 arithmetic, mean
squared error.  Mirrors csrc/costmodel.cu."""
import numpy as np

NF, H = 24, 128
OW1, OB1 = 0, H * NF
OW2 = OB1 + H
OB2 = OW2 + H * H
OW3 = OB2 + H
OB3 = OW3 + H
NP = OB3 + 1


def bf16(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(theta):
    W1 = bf16(theta[OW1:OB1]).reshape(H, NF)
    b1 = theta[OB1:OW2]
    W2 = bf16(theta[OW2:OB2]).reshape(H, H)
    b2 = theta[OB2:OW3]
    W3 = bf16(theta[OW3:OB3])
    b3 = theta[OB3]
    return W1, b1, W2, b2, W3, b3


def forward(theta, X):
    W1, b1, W2, b2, W3, b3 = unpack(theta)
    X = bf16(X)
    a1 = X @ W1.T + b1
    h1 = bf16(np.maximum(a1, 0))
    a2 = h1 @ W2.T + b2
    h2 = bf16(np.maximum(a2, 0))
    y = h2 @ W3 + b3
    return y, (X, h1, h2)


def grad(theta, X, T):
    W1, b1, W2, b2, W3, b3 = unpack(theta)
    y, (Xb, h1, h2) = forward(theta, X)
    n = X.shape[0]
    e = y - T
    dy = (2.0 / n) * e
    g = np.zeros(NP, np.float64)
    g[OW3:OB3] = dy @ h2
    g[OB3] = dy.sum()
    dh2 = np.where(h2 > 0, dy[:, None] * W3[None, :], 0)
    g[OW2:OB2] = (dh2.T @ h1).reshape(-1)
    g[OB2:OW3] = dh2.sum(0)
    dh1 = np.where(h1 > 0, dh2 @ W2, 0)
    g[OW1:OB1] = (dh1.T @ Xb).reshape(-1)
    g[OB1:OW2] = dh1.sum(0)
    return g.astype(np.float32), float((e * e).mean())
