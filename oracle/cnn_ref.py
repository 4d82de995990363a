"""CPU reference of the learned-guess network (numpy, float64).

TEST INFRASTRUCTURE ONLY.  Restates the forward pass and the analytic backward pass
of the four-layer 3x3x3 convolutional network in msg123_b200/csrc/msg_learned.cu
(tap order dz, dy, dx each -1..1, weights W[tap][co][ci], channels-last tensors,
zero padding, GELU(x) = x Phi(x), mean-squared-error loss) so the GPU gradients can be
checked against it.  Inputs and weights are rounded to bfloat16 first, as the GPU
stores them; intermediate activations stay float64 here.
"""
import math

import numpy as np

NCH, NTAP, NLAYER = 16, 27, 4
OFFS = [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(NTAP)]


def bf16(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16          # round to nearest even
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def shift(x, off):
    """y[z,y,x] = x[z+dz, y+dy, x+dx] with zero padding; x has shape (nz, ny, nx, C)."""
    dz, dy, dx = off
    p = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    nz, ny, nx = x.shape[:3]
    return p[1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx]


def conv(x, W, b):
    out = np.zeros(x.shape[:3] + (NCH,))
    for t in range(NTAP):
        out += shift(x, OFFS[t]) @ W[t].T
    return out + b


def conv_t(dz, W):
    """Gradient with respect to the convolution input."""
    dx = np.zeros(dz.shape[:3] + (NCH,))
    for t in range(NTAP):
        dz_, dy_, dx_ = OFFS[t]
        dx += shift(dz @ W[t], (-dz_, -dy_, -dx_))
    return dx


def wgrad(dz, x):
    dW = np.zeros((NTAP, NCH, NCH))
    dzf = dz.reshape(-1, NCH)
    for t in range(NTAP):
        dW[t] = dzf.T @ shift(x, OFFS[t]).reshape(-1, NCH)
    return dW, dzf.sum(0)


def gelu(z):
    return 0.5 * z * (1.0 + np.vectorize(math.erf)(z / math.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + np.vectorize(math.erf)(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)


def loss_and_grad(layers, x, y):
    """layers: [(W[27,16,16], b[16])]; x: (nz, ny, nx, 16); y: (nz, ny, nx)."""
    Ws = [(bf16(W), np.asarray(b, np.float64)) for W, b in layers]
    a = [bf16(x)]
    zs = []
    for l in range(NLAYER):
        z = conv(a[-1], *Ws[l])
        zs.append(z)
        if l < NLAYER - 1:
            a.append(gelu(z))
    out = zs[-1][..., 0]
    n = out.size
    err = out - y
    loss = float(np.mean(err * err))
    dz = np.zeros_like(zs[-1])
    dz[..., 0] = 2.0 * err / n
    grads = [None] * NLAYER
    for l in range(NLAYER - 1, -1, -1):
        dW, db = wgrad(dz, a[l])
        grads[l] = (dW, db)
        if l > 0:
            dz = conv_t(dz, Ws[l][0]) * gelu_d(zs[l - 1])
    return loss, out, grads
