"""numpy restatement of the cost-model MLP (nin -> H -> H -> H -> 1, ReLU,
FP32 weights, mean-squared-error loss) and of its gradients.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA forward/backward kernels
(blasfeo_b200/csrc/mlp.cu); the product never imports it.  Parameter layout
matches the kernels: W1 [nin x H], b1 [H], W2 [H x H], b2, W3 [H x H], b3,
W4 [H x 1], b4 [1], flat and row-major; y = x W + b.
"""
import numpy as np


def unpack(p, nin, H):
    p = np.asarray(p, dtype=np.float64)
    out, o = [], 0
    for shape in [(nin, H), (H,), (H, H), (H,), (H, H), (H,), (H, 1), (1,)]:
        size = int(np.prod(shape))
        out.append(p[o:o + size].reshape(shape))
        o += size
    return out


def forward(p, X, nin, H):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p, nin, H)
    X = np.asarray(X, dtype=np.float64)
    Z1 = X @ W1 + b1
    A1 = np.maximum(Z1, 0)
    Z2 = A1 @ W2 + b2
    A2 = np.maximum(Z2, 0)
    Z3 = A2 @ W3 + b3
    A3 = np.maximum(Z3, 0)
    y = (A3 @ W4 + b4)[:, 0]
    return y, (X, Z1, A1, Z2, A2, Z3, A3)


def loss_and_grad(p, X, t, nin, H):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p, nin, H)
    y, (X, Z1, A1, Z2, A2, Z3, A3) = forward(p, X, nin, H)
    B = len(y)
    d = y - np.asarray(t, dtype=np.float64)
    loss = float(np.mean(d * d))
    dy = (2.0 / B) * d[:, None]
    gW4 = A3.T @ dy
    gb4 = dy.sum(0)
    dZ3 = (dy @ W4.T) * (Z3 > 0)
    gW3 = A2.T @ dZ3
    gb3 = dZ3.sum(0)
    dZ2 = (dZ3 @ W3.T) * (Z2 > 0)
    gW2 = A1.T @ dZ2
    gb2 = dZ2.sum(0)
    dZ1 = (dZ2 @ W2.T) * (Z1 > 0)
    gW1 = X.T @ dZ1
    gb1 = dZ1.sum(0)
    g = np.concatenate([x.ravel() for x in (gW1, gb1, gW2, gb2, gW3, gb3, gW4, gb4)])
    return loss, g
