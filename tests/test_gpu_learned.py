"""Learned Newton initial guess on the GPU.

* GPU forward/backward (tensor-core BF16 convolutions, FP32 accumulation) against the
  float64 numpy reference oracle/cnn_ref.py; the GPU rounds activations and gradients
  to bfloat16 between layers (relative precision 2^-8), hence the 3e-2 bars.
* Training on steps the GPU solver generates lowers the loss.
* The trained network, used as the Newton initial guess, is compared with the plain
  extrapolation and with the reference's start from the previous head.
"""
import numpy as np
import pytest

from msg123_b200.config import make_config
from oracle import cnn_ref

pytestmark = pytest.mark.gpu


def _rand_layers(rng):
    w = []
    for l in range(4):
        W = np.zeros((27, 16, 16), np.float32)
        co = 1 if l == 3 else 16
        ci = 7 if l == 0 else 16
        W[:, :co, :ci] = 0.15 * rng.standard_normal((27, co, ci))
        b = np.zeros(16, np.float32)
        b[:co] = 0.05 * rng.standard_normal(co)
        w.append((W, b))
    return w


def _flat(layers):
    return np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in layers]).astype(np.float32)


def relerr(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


@pytest.mark.parametrize("shape", [(10, 9, 7), (33, 5, 6)])
def test_cnn_gradients_against_reference(shape):
    from msg123_b200.learned import Cnn, unpack
    rng = np.random.default_rng(1)
    nx, ny, nz = shape
    x = np.zeros((nz, ny, nx, 16), np.float32)
    x[..., :7] = rng.standard_normal((nz, ny, nx, 7))
    y = rng.standard_normal((nz, ny, nx)).astype(np.float32)
    layers = _rand_layers(rng)
    cnn = Cnn(seed=3)
    cnn.set_weights(_flat(layers))
    cnn.add_sample(shape, x.reshape(-1, 16), y.reshape(-1))
    loss_g, grad_g, out_g = cnn.loss_grad(0, want_grad=True, want_out=True, n=nx * ny * nz)
    loss_r, out_r, grads_r = cnn_ref.loss_and_grad(layers, x, y)
    assert relerr(out_g, out_r.reshape(-1)) < 3e-2
    assert abs(loss_g - loss_r) / loss_r < 3e-2
    for l, (gW, gb) in enumerate(unpack(grad_g)):
        rW, rb = grads_r[l]
        assert relerr(gW, rW) < 3e-2, l
        assert relerr(gb, rb) < 3e-2, l


@pytest.mark.parametrize("shape", [(10, 9, 7), (33, 5, 6), (130, 4, 3), (256, 6, 5)])
def test_tensor_core_inference_against_reference(shape):
    """The tcgen05 inference path (TMA halo tiles of 128 cells, TMEM accumulators) against
    the float64 reference and against the mma.sync training forward.  Shapes cover a row
    shorter than one tile, a partial second tile and whole tiles."""
    from msg123_b200.learned import Cnn
    rng = np.random.default_rng(7)
    nx, ny, nz = shape
    x = np.zeros((nz, ny, nx, 16), np.float32)
    x[..., :7] = rng.standard_normal((nz, ny, nx, 7))
    y = np.zeros((nz, ny, nx), np.float32)
    layers = _rand_layers(rng)
    cnn = Cnn(seed=3)
    cnn.set_weights(_flat(layers))
    cnn.add_sample(shape, x.reshape(-1, 16), y.reshape(-1))
    out_tc = cnn.infer(0, nx * ny * nz)
    _, _, out_mma = cnn.loss_grad(0, want_grad=False, want_out=True, n=nx * ny * nz)
    _, out_r, _ = cnn_ref.loss_and_grad(layers, x, y)
    assert np.all(np.isfinite(out_tc))
    assert relerr(out_tc, out_r.reshape(-1)) < 3e-2
    assert relerr(out_tc, out_mma) < 1e-2
    cnn.close()


def test_training_lowers_loss():
    from msg123_b200.learned import Cnn, generate
    kw = dict(amg_lag=1, precision=1)
    train = [make_config("hetero", shape=(48, 48, 24), seed=s) for s in (101, 102, 103)]
    cnn = Cnn(seed=0)
    n = generate(cnn, train, steps_per_problem=12, **kw)
    assert n >= 24
    l0 = np.mean([cnn.loss_grad(k, want_grad=False)[0] for k in range(n)])
    cnn.train(iters=600, lr=2e-3, weight_decay=1e-5, seed=1)
    l1 = np.mean([cnn.loss_grad(k, want_grad=False)[0] for k in range(n)])
    print(f"samples {n} loss before {l0:.4e} after {l1:.4e}")
    assert l1 < 0.5 * l0


@pytest.mark.parametrize("shape,seed", [((96, 96, 96), 999), ((128, 128, 96), 998)])
def test_learned_guess_newton_gain(shape, seed):
    """Shipped weights (msg123_b200/train_guess.py: 20,000 steps generated on 128x128x96
    fields of seeds 5000-5399, rain and drainage) on held-out fields of the same generator:
    Newton iterations per step over 24 steps from the reference's previous-head start, from
    the plain extrapolation and from the learned guess (used directly, extrapolation
    fallback), the value path's other settings alike."""
    from msg123_b200.learned import Cnn, newton_per_step
    from msg123_b200.train_guess import load
    kw = dict(amg_lag=4, precision=1, vg_form=1, jv_mode=1, guess_select=0)
    cnn = load(Cnn(seed=0))
    test = make_config("hetero", shape=shape, seed=seed, sigma=1.5)
    n0, s0, _ = newton_per_step(test, 24, guess_mode=0, **kw)
    n1, s1, _ = newton_per_step(test, 24, guess_mode=1, **kw)
    n2, s2, fb = newton_per_step(test, 24, cnn=cnn, guess_mode=2, **kw)
    print(f"{shape} Newton/step previous-head {n0:.2f} ({s0['current_t']:.0f} s) extrapolation {n1:.2f} "
          f"({s1['current_t']:.0f} s) learned {n2:.2f} ({s2['current_t']:.0f} s) (fallbacks, rejected {fb})")
    assert s2["accepted"] == 24
    assert n1 < n0
    assert n2 < n1                 # the network improves on the plain extrapolation
