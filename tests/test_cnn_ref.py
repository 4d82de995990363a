"""Pins the numpy reference of the learned-guess network (no GPU needed): its analytic
gradients match central finite differences in float64, its convolution matches the
definition written out as loops, and its bfloat16 rounding matches torch's."""
import numpy as np

from oracle import cnn_ref


def test_reference_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    shape = (3, 4, 3)
    x = np.zeros(shape + (16,))
    x[..., :7] = rng.standard_normal(shape + (7,))
    x = cnn_ref.bf16(x)
    y = rng.standard_normal(shape)
    layers = []
    for l in range(4):
        W = np.zeros((27, 16, 16))
        co = 1 if l == 3 else 16
        ci = 7 if l == 0 else 16
        W[:, :co, :ci] = cnn_ref.bf16(0.2 * rng.standard_normal((27, co, ci)))
        b = np.zeros(16)
        b[:co] = 0.1 * rng.standard_normal(co)
        layers.append((W, b))
    loss, out, grads = cnn_ref.loss_and_grad(layers, x, y)
    # the reference rounds weights to bf16; probe along directions it keeps exact by
    # perturbing the biases and checking weight gradients on an unrounded copy
    def loss_of(ls):
        saved = cnn_ref.bf16
        cnn_ref.bf16 = lambda a: np.asarray(a, dtype=np.float64)
        try:
            return cnn_ref.loss_and_grad(ls, x, y)[0]
        finally:
            cnn_ref.bf16 = saved
    base = loss_of(layers)
    assert abs(base - loss) <= 1e-12 * max(1.0, abs(loss))
    eps = 1e-6
    for l, (tap, co, ci) in [(0, (13, 2, 3)), (1, (0, 5, 7)), (2, (26, 15, 0)), (3, (4, 0, 9))]:
        ls = [(W.copy(), b.copy()) for W, b in layers]
        ls[l][0][tap, co, ci] += eps
        up = loss_of(ls)
        ls[l][0][tap, co, ci] -= 2 * eps
        dn = loss_of(ls)
        fd = (up - dn) / (2 * eps)
        assert abs(fd - grads[l][0][tap, co, ci]) <= 1e-6 * max(1e-3, abs(fd))
    for l in range(4):
        ls = [(W.copy(), b.copy()) for W, b in layers]
        ls[l][1][0] += eps
        up = loss_of(ls)
        ls[l][1][0] -= 2 * eps
        dn = loss_of(ls)
        assert abs((up - dn) / (2 * eps) - grads[l][1][0]) <= 1e-6 * max(1e-3, abs(grads[l][1][0]))


def test_conv_matches_a_direct_loop():
    """The reference convolution against the definition written out as loops: tap t is
    (dz, dy, dx) = (t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1), W[t][co][ci], zero padding."""
    rng = np.random.default_rng(4)
    nz, ny, nx = 3, 4, 5
    x = rng.standard_normal((nz, ny, nx, 16))
    W = rng.standard_normal((27, 16, 16))
    b = rng.standard_normal(16)
    out = cnn_ref.conv(x, W, b)
    ref = np.zeros_like(out)
    for z in range(nz):
        for y in range(ny):
            for xx in range(nx):
                acc = b.copy()
                for t in range(27):
                    dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
                    zz, yy, xs = z + dz, y + dy, xx + dx
                    if 0 <= zz < nz and 0 <= yy < ny and 0 <= xs < nx:
                        acc += W[t] @ x[zz, yy, xs]
                ref[z, y, xx] = acc
    assert np.max(np.abs(out - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_bf16_rounding_is_nearest_even():
    """cnn_ref.bf16 against torch's float32 -> bfloat16 conversion (round to nearest, ties
    to even), including exact ties and values near the overflow of the exponent."""
    import torch
    rng = np.random.default_rng(5)
    a = np.concatenate([rng.standard_normal(10000).astype(np.float32),
                        np.array([1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -1.0 - 2.0 ** -8, 0.0, -0.0,
                                  3.3895e38, 1e-40], dtype=np.float32)])
    want = torch.from_numpy(a).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(cnn_ref.bf16(a), want)


def test_shipped_weights_are_well_formed():
    """The committed network (msg123_b200/weights/guess_cnn.npy): one float32 vector of the
    four layers' taps and biases, finite, and the float64 reference runs it on a small
    grid to a finite output."""
    import os
    from msg123_b200.learned import unpack
    w = np.load(os.path.join(os.path.dirname(__file__), "..", "msg123_b200", "weights", "guess_cnn.npy"))
    assert w.dtype == np.float32 and w.shape == (4 * (27 * 16 * 16 + 16),)
    assert np.all(np.isfinite(w))
    layers = [(cnn_ref.bf16(W), b.astype(np.float64)) for W, b in unpack(w)]
    x = np.zeros((3, 4, 5, 16))
    x[..., :7] = cnn_ref.bf16(np.random.default_rng(6).standard_normal((3, 4, 5, 7)))
    _, out, _ = cnn_ref.loss_and_grad(layers, x, np.zeros((3, 4, 5)))
    assert np.all(np.isfinite(out))
