"""CPU FP64 restatement of the bracket-predictor network (test infrastructure: the gradient and
forward oracle for the engine's tensor-core kernels; nothing here is used by the engine).

Network: 6 -> 128 -> 128 -> 128 -> 3, SiLU after the three hidden layers, weights row-major
[out][in], flat parameter vector in the order W1, b1, W2, b2, W3, b3, W4, b4.  Loss: masked mean
squared error sum(m (y - t)^2) / sum(m).

With bf16=True the operands that the engine feeds to its BF16 tensor cores are rounded to bfloat16
(round to nearest even) at the same places: the hidden activations h1, h2 and the weights W2, W3 in
the forward products, and the back-propagated dz2, dz3 in the backward products.  Everything else,
as on the engine, stays in higher precision (here FP64).
"""
import numpy as np

SIZES = [(128, 6), (128, 128), (128, 128), (3, 128)]


def num_params():
    return sum(o * i + o for o, i in SIZES)


def unpack(p):
    out, k = [], 0
    for o, i in SIZES:
        W = p[k:k + o * i].reshape(o, i)
        k += o * i
        b = p[k:k + o]
        k += o
        out.append((W, b))
    return out


def pack(layers):
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in layers])


def bf16(a):
    """round to bfloat16 (nearest even) and back, through float32"""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1 + np.exp(-z))


def dsilu(z):
    s = 1 / (1 + np.exp(-z))
    return s * (1 + z * (1 - s))


def forward(p, x, bf=False):
    r = bf16 if bf else (lambda a: a)
    (W1, b1), (W2, b2), (W3, b3), (W4, b4) = unpack(np.asarray(p, dtype=np.float64))
    z1 = x @ W1.T + b1
    h1 = silu(z1)
    z2 = r(h1) @ r(W2).T + b2
    h2 = silu(z2)
    z3 = r(h2) @ r(W3).T + b3
    h3 = silu(z3)
    y = h3 @ W4.T + b4
    return y, (z1, h1, z2, h2, z3, h3)


def loss_grad(p, x, t, m, bf=False):
    """loss and its gradient with respect to the flat parameter vector"""
    r = bf16 if bf else (lambda a: a)
    p = np.asarray(p, dtype=np.float64)
    (W1, b1), (W2, b2), (W3, b3), (W4, b4) = unpack(p)
    y, (z1, h1, z2, h2, z3, h3) = forward(p, x, bf)
    S = max(float(np.sum(m)), 1.0)
    loss = float(np.sum(m * (y - t) ** 2) / S)
    dy = 2 * m * (y - t) / S
    dW4, db4 = dy.T @ h3, dy.sum(0)
    dz3 = (dy @ W4) * dsilu(z3)
    dW3, db3 = r(dz3).T @ r(h2), dz3.sum(0)
    dz2 = (r(dz3) @ r(W3)) * dsilu(z2)
    dW2, db2 = r(dz2).T @ r(h1), dz2.sum(0)
    dz1 = (r(dz2) @ r(W2)) * dsilu(z1)
    dW1, db1 = dz1.T @ x, dz1.sum(0)
    return loss, pack([(dW1, db1), (dW2, db2), (dW3, db3), (dW4, db4)])
