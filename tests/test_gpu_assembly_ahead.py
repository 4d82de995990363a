"""The line search's assembly ahead (run_backtr in msg_api.cu: the residual evaluation at the
full Newton step is the assembly pass, whose system the next Newton iteration uses) changes
no value.  With the phase timers on, the library takes the plain path (residual pass in the
line search, assembly at the next iteration); both runs give the same heads bit for bit and
the same Newton, Krylov and backtracking counts, on the mixed AMG path (where the line
search also backtracks, which drops the system assembled ahead) and on the FP64 DILU path."""
import numpy as np
import pytest

from msg123_b200.config import make_config

pytestmark = pytest.mark.gpu

CASES = [
    ("hetero", dict(shape=(40, 36, 20), seed=5),
     dict(precision=1, precon_type=1, ref_quirks=0, amg_coarse_max=200, amg_lag=4, vg_form=1, jv_mode=1,
          sim_type=0, inc_fact=1.0, ini_step=1800.0, criteria=1e-8, maxout_iter=60)),
    ("box", dict(shape=(10, 9, 12), nsteps=4), dict()),
]


@pytest.mark.parametrize("name,pkw,skw", CASES)
def test_assembly_ahead_same_bits(name, pkw, skw):
    from msg123_b200.solver import GpuSolver
    p = make_config(name, **pkw)
    res = []
    for timing in (False, True):
        g = GpuSolver(p, **skw)
        g.set_timing(timing)
        g.init_state()
        rc, st = g.advance(nsteps=4)
        assert rc == 0
        res.append((g.get_state()["head_new"].copy(),
                    (st["accepted"], st["newton_total"], st["krylov_total"], st["back_total"])))
        g.close()
    print(name, res[0][1], res[1][1])
    assert res[0][1] == res[1][1]
    assert np.array_equal(res[0][0], res[1][0])
