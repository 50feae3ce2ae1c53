"""CPU reference (TEST INFRASTRUCTURE ONLY) of the learned coarse-correction network.

The network has no counterpart in the reference; this numpy restatement is the only pin
of the hand-written CUDA forward/backward kernels (gale_b200/csrc/gg_learned.cu), used
by tests/test_learned.py for the gradient check.

Layout (same as the device): tensors [batch][channel][node] over the nodal grid of one
multigrid level, node index x-fastest; 3^dim stencils with zero padding; weights
W1[c_out][tap][c_in], b1[c_out], W2[c_out][tap][c_in], b2[c_out], tap = (dx+1) + 3(dy+1)
(+ 9(dz+1)).  Forward: h = relu(conv(x, W1) + b1), y = conv(h, W2) + b2.  Loss:
Σ_b ‖m ⊙ (y_b − t_b)‖² / ‖m ⊙ t_b‖² with the free-dof mask m of the output channels.
"""
from __future__ import annotations

import numpy as np


def taps(dim):
    out = []
    for dz in ((-1, 0, 1) if dim == 3 else (0,)):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                out.append((dx, dy, dz))
    return out


def shift(a, grid, d):
    """b[n] = a[n + d] with zeros outside (a: [..., nodes])."""
    nx, ny, nz = grid
    A = a.reshape(a.shape[:-1] + (nz, ny, nx))
    B = np.zeros_like(A)
    dx, dy, dz = d
    src = [slice(max(0, k), n + min(0, k)) for k, n in ((dz, nz), (dy, ny), (dx, nx))]
    dst = [slice(max(0, -k), n + min(0, -k)) for k, n in ((dz, nz), (dy, ny), (dx, nx))]
    B[(Ellipsis,) + tuple(dst)] = A[(Ellipsis,) + tuple(src)]
    return B.reshape(a.shape)


def conv(x, W, b, grid, dim):
    """x [B][Cin][N], W [Cout][T][Cin] → [B][Cout][N]."""
    out = np.zeros((x.shape[0], W.shape[0], x.shape[2]), dtype=np.float64)
    for t, d in enumerate(taps(dim)):
        xs = shift(x, grid, d)
        out += np.einsum("oc,bcn->bon", W[:, t, :], xs)
    return out + b[None, :, None]


def conv_bwd(x, dout, W, grid, dim):
    """grads of conv w.r.t. W, b and x."""
    dW = np.zeros_like(W, dtype=np.float64)
    dx = np.zeros_like(x, dtype=np.float64)
    for t, d in enumerate(taps(dim)):
        xs = shift(x, grid, d)
        dW[:, t, :] = np.einsum("bon,bcn->oc", dout, xs)
        back = np.einsum("oc,bon->bcn", W[:, t, :], dout)
        dx += shift(back, grid, (-d[0], -d[1], -d[2]))
    db = dout.sum(axis=(0, 2))
    return dW, db, dx


def forward_backward(x, target, mask, W1, b1, W2, b2, grid, dim):
    z1 = conv(x, W1, b1, grid, dim)
    h = np.maximum(z1, 0.0)
    y = conv(h, W2, b2, grid, dim)
    m = mask[None, :, :]
    wgt = 1.0 / np.maximum((m * target ** 2).sum(axis=(1, 2)), 1e-300)
    res = m * (y - target)
    loss = float((wgt * (res ** 2).sum(axis=(1, 2))).sum())
    dy = 2.0 * wgt[:, None, None] * res
    dW2, db2, dh = conv_bwd(h, dy, W2, grid, dim)
    dz1 = dh * (z1 > 0)
    dW1, db1, _ = conv_bwd(x, dz1, W1, grid, dim)
    return y, loss, (dW1, db1, dW2, db2)
