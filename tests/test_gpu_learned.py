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


def _to_end(problem, T, cnn=None, **kw):
    """Accepted steps, Newton iterations, rejected steps and guess statistics of one run from
    the hydrostatic start to the simulated time T (the last step is clipped to T)."""
    from msg123_b200.solver import GpuSolver
    with GpuSolver(problem, end_time=T, **kw) as g:
        if cnn is not None:
            cnn.attach(g)
        g.init_state()
        steps = newton = rejected = 0
        while True:
            rc, st = g.advance(nsteps=1)
            assert rc == 0
            steps += st["accepted"]
            newton += st["newton_total"]
            rejected += st["rejected"]
            if st["current_t"] >= T or steps > 400:
                break
        out = dict(t=st["current_t"], steps=steps, newton=newton, rejected=rejected,
                   fallbacks=g.guess_fallbacks(), not_used=g.guess_rejected())
        if cnn is not None:
            cnn.detach(g)
    return out


def test_learned_guess_newton_gain():
    """Shipped weights (msg123_b200/train_guess.py: 20,000 steps generated on 128x128x96
    fields of seeds 5000-5399, sigma_lnK 0.5-1.5, rain and drainage) on a held-out field of
    the same generator, run from the hydrostatic start to 10,000 s simulated (rain and the
    drainage that follows it): Newton iterations in total from the plain extrapolation, from
    the learned guess used directly (guess_select 0) and from the vetted learned guess
    (guess_select 2: the network's guess is kept only when its residual norm is below the
    extrapolation's; after a loss it is skipped for 1, 2, 4, 8 steps).  The value path's
    other settings alike.  Measured: extrapolation 340, vetted 317 (29 steps against 31)."""
    from msg123_b200.learned import Cnn
    from msg123_b200.train_guess import load
    kw = dict(amg_lag=4, precision=1, vg_form=1, jv_mode=1)
    cnn = load(Cnn(seed=0))
    p = make_config("hetero", shape=(128, 128, 96), seed=998, sigma=1.5)
    T = 10000.0
    ex = _to_end(p, T, guess_mode=1, **kw)
    direct = _to_end(p, T, cnn=cnn, guess_mode=2, guess_select=0, **kw)
    vetted = _to_end(p, T, cnn=cnn, guess_mode=2, guess_select=2, **kw)
    print(f"to {T:.0f} s: extrapolation {ex}\n  learned, direct {direct}\n  learned, vetted {vetted}")
    for r in (ex, direct, vetted):
        assert r["t"] == pytest.approx(T)
    assert vetted["newton"] < ex["newton"]     # the vetted network improves on the plain extrapolation
    cnn.close()
