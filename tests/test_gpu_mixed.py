"""Mixed precision (precision = 1): FP32 V-cycle smoothers and level-1 operator, BF16
coarse-level off-diagonals, FP64 coarsest inverse, FP64 BiCGStab and Newton.

The FP64 oracle is the reference for head and mass balance: a mixed-precision run must
land within the headline tolerances of the plain FP64 solution on the same inputs."""
import numpy as np
import pytest

from msg123_b200.config import make_config
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

AMG = dict(precon_type=1, ref_quirks=0, amg_coarse_max=200)


def test_mixed_vcycle_close_to_fp64():
    from msg123_b200.solver import GpuSolver
    p = make_config("hetero", shape=(32, 28, 18), seed=3)
    o = Oracle(p, **AMG)
    o.init_state()
    o.set_state(head_new=p.head0 + 0.004 * np.random.default_rng(3).standard_normal(p.ncalc), delt=3600.0)
    d, lu, r = o.make_matvec()
    o.set_system(d, lu, r)
    g = GpuSolver(p, precision=1, **AMG)
    g.set_system(d, lu, r)
    v = np.random.default_rng(5).standard_normal(p.ncalc)
    zg, zo = g.precond(v), o.precond(v)
    assert np.linalg.norm(zg - zo) / np.linalg.norm(zo) < 2e-2


def _run_pair(lag, vg_form=0):
    from msg123_b200.solver import GpuSolver
    p = make_config("hetero", shape=(32, 28, 16), seed=12)
    ov = dict(AMG, sim_type=0, inc_fact=1.0, ini_step=1800.0, amg_lag=lag, criteria=1e-8, maxout_iter=60)
    g, o = GpuSolver(p, precision=1, vg_form=vg_form, **ov), Oracle(p, **ov)
    t = Oracle(p, **dict(ov, amg_lag=1, criteria=1e-11))
    g.init_state(); o.init_state(); t.init_state()
    rg, sg = g.advance(nsteps=3)
    ro, so = o.advance(nsteps=3)
    rt, stt = t.advance(nsteps=3)
    assert rg == ro == rt == 0
    assert sg["rejected"] == so["rejected"] == 0 and sg["current_t"] == so["current_t"] == stt["current_t"]
    hg, ho, ht = g.get_state()["head_new"], o.get_state()["head_new"], t.get_state()["head_new"]
    rel = lambda a, b: float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    mg, mo = g.calc_mass(), o.calc_mass()
    print("mixed", sg, "fp64 oracle", so, "head err vs oracle", rel(hg, ho), "vs criteria 1e-11", rel(hg, ht),
          "oracle vs 1e-11", rel(ho, ht))
    return rel(hg, ho), rel(hg, ht), np.max(np.abs(mg - mo)) / abs(mo[2])


@pytest.mark.parametrize("lag,vg_form", [(1, 0), (4, 0), (4, 1), (0, 0)])
def test_mixed_run_matches_fp64_oracle(lag, vg_form):
    """Mixed precision changes the Newton path, so the mixed run and an FP64 run agree to
    the accuracy of their common stopping test (max|dh| <= 1e-8 max|h|), not bit for bit.
    The mixed run is held to 1e-8 of the FP64 oracle's solution at criteria 1e-11 (the
    converged answer of the time steps).  Where the two paths stay together the FP64
    oracle's own run at criteria 1e-8 is within 1e-8 of the mixed run too, and the step
    volumes within 1e-10 of the inflow; with the hierarchy rebuilt at every Newton iteration
    (lag 0) the FP64 run settles seepage cells after 22 backtracks and stops 2.4e-8 from the
    converged answer -- its own stopping rule's slack -- while the mixed run stays within
    9e-9 of it, so only the comparison with the converged answer applies there.  vg_form = 1
    (the two-pow kr of the value path) runs against the oracle's reference form."""
    err, err_tight, merr = _run_pair(lag, vg_form)
    assert err_tight <= 1e-8
    if lag != 0:
        assert err <= 1e-8
        assert merr <= 1e-10
