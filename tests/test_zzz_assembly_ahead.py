"""The line search's assembly ahead (run_backtr in msg_api.cu: the residual evaluation at the
full Newton step is the assembly pass, whose system the next Newton iteration uses) changes
no value.  With the phase timers on, the library takes the plain path (residual pass in the
line search, assembly at the next iteration); both runs give the same heads bit for bit and
the same Newton, Krylov and backtracking counts, on the mixed AMG path (a backtracking
line search drops the system assembled ahead) and on the FP64 DILU path."""
import numpy as np
import pytest

from msg123_b200.config import make_config

pytestmark = pytest.mark.gpu

# the mixed run of test_gpu_mixed.py (lag 4, two-pow kr) plus the line-search
# slope from BiCGStab, and the config-1 box (FP64, BiCGStab + DILU, finite-difference J dh)
CASES = [
    ("hetero", dict(shape=(32, 28, 16), seed=12), 3,
     dict(precision=1, precon_type=1, ref_quirks=0, amg_coarse_max=200, amg_lag=4, vg_form=1, jv_mode=1,
          sim_type=0, inc_fact=1.0, ini_step=1800.0, criteria=1e-8, maxout_iter=60)),
    ("box", dict(), 6, dict()),
]


@pytest.mark.parametrize("name,pkw,nsteps,skw", CASES)
def test_assembly_ahead_same_bits(name, pkw, nsteps, skw):
    from msg123_b200.solver import GpuSolver
    p = make_config(name, **pkw)
    res = []
    for timing in (False, True):
        g = GpuSolver(p, **skw)
        g.set_timing(timing)
        g.init_state()
        rc, st = g.advance(nsteps=nsteps)
        assert rc == 0
        res.append((g.get_state()["head_new"].copy(),
                    (st["accepted"], st["newton_total"], st["krylov_total"], st["back_total"])))
        g.close()
    print(name, res[0][1], res[1][1])
    assert res[0][1] == res[1][1]
    assert np.array_equal(res[0][0], res[1][0])
