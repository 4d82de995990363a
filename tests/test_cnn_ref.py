"""Pins the numpy reference of the learned-guess network: its analytic gradients must
match central finite differences in float64 (no GPU needed)."""
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
