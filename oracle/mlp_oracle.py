"""FP64 numpy restatement of the learned self-energy update's network (test infrastructure).

The network has no counterpart in CoQui (its loop knows only damping and DIIS,
src/numerics/iter_scf); this file is the CPU oracle that the device forward and backward
kernels are checked against.  Layout of the flat parameter vector: W1 (width, in), b1,
W2 (width, width), b2, W3 (out, width), b3.  The device runs the forward pass with BF16
copies of the parameters, so the oracle rounds them the same way (round to nearest even) and
differentiates through the rounding as the identity.
"""
import numpy as np


def bf16_round(x):
    """float32 -> nearest bfloat16 (ties to even), returned as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (u & 0xFFFFFFFF).astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p, din, width, dout):
    p = np.asarray(p, np.float64)
    o = 0
    shapes = [(width, din), (width,), (width, width), (width,), (dout, width), (dout,)]
    out = []
    for sh in shapes:
        n = int(np.prod(sh))
        out.append(p[o:o + n].reshape(sh))
        o += n
    assert o == p.size
    return out


def forward(p, X, din, width, dout, round_params=True):
    rnd = bf16_round if round_params else (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, W3, b3 = [rnd(a) for a in unpack(p, din, width, dout)]
    X = np.asarray(X, np.float64)
    h1 = np.tanh(X @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ W3.T + b3, (X, h1, h2, W1, W2, W3)


def loss_and_grad(p, X, T, din, width, dout, round_params=True):
    """Mean squared error over the batch and outputs, and its gradient (flat, like p)."""
    Y, (X, h1, h2, W1, W2, W3) = forward(p, X, din, width, dout, round_params)
    T = np.asarray(T, np.float64)
    n = Y.size
    dY = 2.0 * (Y - T) / n
    gW3 = dY.T @ h2
    gb3 = dY.sum(0)
    dz2 = (dY @ W3) * (1.0 - h2 ** 2)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * (1.0 - h1 ** 2)
    gW1 = dz1.T @ X
    gb1 = dz1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return float(((Y - T) ** 2).mean()), g
