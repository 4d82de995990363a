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


def _run_pair(lag, crit, vg_form=0):
    from msg123_b200.solver import GpuSolver
    p = make_config("hetero", shape=(32, 28, 16), seed=12)
    ov = dict(AMG, sim_type=0, inc_fact=1.0, ini_step=1800.0, amg_lag=lag, criteria=crit, maxout_iter=60)
    g, o = GpuSolver(p, precision=1, vg_form=vg_form, **ov), Oracle(p, **ov)
    g.init_state(); o.init_state()
    rg, sg = g.advance(nsteps=3)
    ro, so = o.advance(nsteps=3)
    assert rg == ro == 0
    assert sg["rejected"] == so["rejected"] == 0 and sg["current_t"] == so["current_t"]
    hg, ho = g.get_state()["head_new"], o.get_state()["head_new"]
    err = np.max(np.abs(hg - ho)) / np.max(np.abs(ho))
    mg, mo = g.calc_mass(), o.calc_mass()
    print("mixed", sg, "fp64 oracle", so, "head err", err)
    return err, np.max(np.abs(mg - mo)) / abs(mo[2])


@pytest.mark.parametrize("lag,bound,vg_form", [(1, 1e-8, 0), (4, 1e-8, 0), (4, 1e-8, 1), (0, 3e-8, 0)])
def test_mixed_run_matches_fp64_oracle(lag, bound, vg_form):
    """Mixed precision changes the Newton path, so the two runs agree to the accuracy of
    their common stopping test (max|dh| <= 1e-8 max|h|), not bit for bit.  With the
    hierarchy kept per time step (amg_lag >= 1) the heads agree to ~1e-10.  Rebuilding the
    AMG at every Newton iteration (amg_lag = 0) lets the two paths settle a few top cells
    on different sides of the seepage-face switch (h = surf_top, where the surface term
    of calc_func is not differentiable), which leaves a gap of ~1.5e-8 that a tighter
    Newton tolerance does not remove; that case is bounded at 3x the tolerance.  Mass
    balance agrees within 1e-10 of the inflow in every case.  vg_form = 1 (the two-pow
    kr of the value path) runs against the oracle's reference form."""
    err, merr = _run_pair(lag, 1e-8, vg_form)
    assert err <= bound
    assert merr <= 1e-10
