"""numpy restatement of the sensor network's forward pass, loss and gradient.

TEST INFRASTRUCTURE: checks the library's hand-written forward/backward
kernel (cbns_mlp_grad) in FP64.  Layout: W1[32][15] b1[32] W2[32][32] b2[32]
w3[32] b3; loss = mean over samples of -w (y log p + (1-y) log(1-p)),
p = sigmoid(logit), w = pos_weight for y = 1 else 1.
"""
import numpy as np


def unpack(P):
    P = np.asarray(P, dtype=np.float64)
    return (P[0:480].reshape(32, 15), P[480:512], P[512:1536].reshape(32, 32), P[1536:1568], P[1568:1600], P[1600])


def forward(P, X):
    W1, b1, W2, b2, w3, b3 = unpack(P)
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0)
    return h2 @ w3 + b3, (a1, h1, a2, h2)


def loss_grad(P, X, Y, pos_weight=1.0):
    X = np.asarray(X, dtype=np.float64)
    y = np.asarray(Y, dtype=np.float64)
    W1, b1, W2, b2, w3, b3 = unpack(P)
    z, (a1, h1, a2, h2) = forward(P, X)
    n = X.shape[0]
    w = np.where(y > 0, pos_weight, 1.0)
    lp = -np.log1p(np.exp(-np.abs(z))) + np.minimum(z, 0)
    loss = -np.sum(w * (y * lp + (1 - y) * (lp - z))) / n
    p = 1 / (1 + np.exp(-z))
    dz = w * (p - y) / n
    g = np.zeros(1601)
    g[1568:1600] = h2.T @ dz
    g[1600] = dz.sum()
    g2 = np.outer(dz, w3) * (a2 > 0)
    g[512:1536] = (g2.T @ h1).reshape(-1)
    g[1536:1568] = g2.sum(0)
    g1 = (g2 @ W2) * (a1 > 0)
    g[0:480] = (g1.T @ X).reshape(-1)
    g[480:512] = g1.sum(0)
    return loss, g
