"""Failure detection and recovery, made on the host (no GPU fault, trap or hang).

* NaN in the state: Newton reports MSG_NAN (Nonlinear_solution.f90:151-155) -- oracle and GPU.
* Newton cap: with maxout_iter too small for the first step the time loop rolls the state
  back and halves dt (Time_module.f90:253-264) until steps are accepted; the GPU takes the
  same decisions as the oracle.
* dt floor: a state that can never converge (NaN) is rejected at every dt until dt falls
  below DSMAL, and the time loop ends with MSG_DT_TOO_SMALL (Time_module.f90:72-73).
* Learned guess: a network with garbage weights is either rejected by the residual check
  (guess_select = 1) or, used anyway (guess_select = 0), fails and falls back to the plain
  extrapolation; both runs end where the extrapolation run ends.
* Bounded waits of the tensor-core kernel: the input box of one tile is withheld, the wait
  on it runs out after about a second, the kernel drains and returns, and the host gets an
  error status while the context stays usable.
"""
import numpy as np
import pytest

from msg123_b200.config import make_config

MSG_OK, MSG_NEWTON_MAXIT, MSG_NAN, MSG_DT_TOO_SMALL = 0, 1, 2, 5


def relmax(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _nan_problem():
    p = make_config("box", shape=(6, 5, 8), nsteps=2)
    h = p.head0.copy()
    h[17] = np.nan
    return p, h


def test_oracle_nan_state():
    from oracle.oracle import Oracle
    p, h = _nan_problem()
    o = Oracle(p)
    o.init_state()
    o.set_state(head_new=h, head_old=h, delt=1800.0)
    rc, st = o.calc_numsol()
    assert rc == MSG_NAN


def test_oracle_newton_cap_rolls_back_and_halves_dt():
    from oracle.oracle import Oracle
    p = make_config("box", shape=(6, 5, 8), nsteps=3, maxout_iter=2)
    o = Oracle(p)
    o.init_state()
    rc, st = o.advance(nsteps=3)
    assert rc == MSG_OK and st["accepted"] == 3 and st["rejected"] >= 1
    # each rejection halves dt; inc_fact = 1 keeps it there once steps are accepted
    assert st["delt"] == pytest.approx(1800.0 * 0.5 ** st["rejected"])


def test_oracle_dt_floor():
    from oracle.oracle import Oracle
    p, h = _nan_problem()
    o = Oracle(p)
    o.init_state(head=h)
    rc, st = o.advance(nsteps=1)
    assert rc == MSG_DT_TOO_SMALL and st["accepted"] == 0 and st["rejected"] > 10


@pytest.mark.gpu
def test_gpu_nan_state():
    from msg123_b200.solver import GpuSolver
    p, h = _nan_problem()
    g = GpuSolver(p)
    g.init_state()
    g.set_state(head_new=h, head_old=h, delt=1800.0)
    rc, st = g.calc_numsol()
    assert rc == MSG_NAN
    # the context stays usable: a clean state converges again
    g.init_state()
    rc, st = g.advance(nsteps=1)
    assert rc == MSG_OK and st["accepted"] == 1


@pytest.mark.gpu
def test_gpu_newton_cap_matches_oracle():
    from msg123_b200.solver import GpuSolver
    from oracle.oracle import Oracle
    p = make_config("box", shape=(6, 5, 8), nsteps=3, maxout_iter=2)
    g, o = GpuSolver(p), Oracle(p)
    g.init_state()
    o.init_state()
    rg, sg = g.advance(nsteps=3)
    ro, so = o.advance(nsteps=3)
    assert rg == ro == MSG_OK
    assert sg["rejected"] == so["rejected"] >= 1
    assert sg["delt"] == so["delt"] and sg["current_t"] == so["current_t"]
    assert relmax(g.get_state()["head_new"], o.get_state()["head_new"]) <= 1e-8


@pytest.mark.gpu
def test_gpu_dt_floor():
    from msg123_b200.solver import GpuSolver
    p, h = _nan_problem()
    g = GpuSolver(p)
    g.init_state(head=h)
    rc, st = g.advance(nsteps=1)
    assert rc == MSG_DT_TOO_SMALL and st["accepted"] == 0 and st["rejected"] > 10


def _garbage_cnn(seed=5):
    from msg123_b200.learned import Cnn
    cnn = Cnn(seed=0)
    rng = np.random.default_rng(seed)
    cnn.set_weights((3.0 * rng.standard_normal(cnn.nparam)).astype(np.float32))
    cnn.set_deadband(0.0)
    return cnn


@pytest.mark.gpu
@pytest.mark.parametrize("select", [1, 0])
def test_gpu_bad_learned_guess_is_contained(select):
    """A garbage network must not change the result: rejected by the residual check
    (guess_select = 1) or replaced by the extrapolation after Newton fails on it
    (guess_select = 0).  amg_lag = 0 so that a failed attempt leaves no AMG state behind."""
    from msg123_b200.solver import GpuSolver
    p = make_config("hetero", shape=(32, 24, 16), seed=11)
    kw = dict(precision=1, amg_lag=0, maxout_iter=8)
    ref = GpuSolver(p, guess_mode=1, **kw)
    ref.init_state()
    rr, sr = ref.advance(nsteps=6)
    g = GpuSolver(p, guess_mode=2, guess_select=select, **kw)
    cnn = _garbage_cnn()
    cnn.attach(g)
    g.init_state()
    rg, sg = g.advance(nsteps=6)
    assert rr == rg == MSG_OK
    fallbacks, rejected = g.guess_fallbacks(), g.guess_rejected()
    if select:
        assert rejected >= 4 and fallbacks == 0
    else:
        assert fallbacks >= 1
    assert sg["current_t"] == sr["current_t"]
    assert relmax(g.get_state()["head_new"], ref.get_state()["head_new"]) <= 1e-12
    cnn.close()


@pytest.mark.gpu
def test_gpu_tensor_core_wait_runs_out_and_reports():
    from msg123_b200.learned import Cnn
    rng = np.random.default_rng(3)
    shape = (64, 32, 6)
    n = int(np.prod(shape))
    cnn = Cnn(seed=1)
    cnn.add_sample(shape, rng.standard_normal((n, 16)).astype(np.float32), np.zeros(n, np.float32))
    good = cnn.infer(0, n)
    rc, msg = cnn.infer_withhold(0, n, tile=3)
    assert rc != 0 and "bounded wait" in msg
    # the device is still usable and the next pass is correct
    again = cnn.infer(0, n)
    assert np.array_equal(good, again)
    cnn.close()
