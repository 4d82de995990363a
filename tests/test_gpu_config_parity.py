"""Parity at the benchmarked configurations: the GPU against the oracle on the workloads
and settings the benchmark measures, not only on small grids.

* the 256x256x64 heterogeneous block (4,194,304 cells) on the plain FP64 path
  (BiCGStab + AMG rebuilt at every Newton iteration, Newton from the previous head,
  adaptive dt from 600 s) over its first four accepted steps;
* the value path of the benchmark (mixed precision, learned initial guess with the
  shipped weights, AMG kept for 12 steps, two-pow kr, slope from BiCGStab's residual) on
  a 1,048,576-cell block of the 25.2M-cell workload's generator (sigma_lnK = 1.5) over
  twelve steps, against the FP64 oracle solved to a 1000x tighter Newton tolerance at the
  same simulated times (the time step grows by a fixed factor, so both runs meet at the
  same times whatever their Newton counts);
* the reference's own AMG mode (precon_type = 1, ref_quirks = 1: the preconditioner acts
  as the level-1 DILU and the line-search slope reads its last input) over adaptive steps;
* three members of the batched ensemble, advanced together, each against the oracle.

Bars: head max|h_gpu - h_ref| / max|h_ref| <= 1e-8; mass: the step volumes of the two runs
within 1e-10 of the inflow volume, and each step's mass balance closing to 1e-10 of it;
Newton and Krylov counts printed.
"""
import numpy as np
import pytest

from msg123_b200.config import make_config, make_member
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

HEAD_TOL = 1e-8
PLAIN = dict(precon_type=1, ref_quirks=0, precision=0, amg_lag=0, guess_mode=0, vg_form=0)
VALUE = dict(precon_type=1, ref_quirks=0, precision=1, amg_lag=12, guess_mode=2, guess_select=0, vg_form=1,
             jv_mode=1)


def relmax(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def closure(m):
    """Mass-balance residual of one step's volumes (storage, flow, recharge, well, surface,
    river, lake, sea, drainage): storage change minus every inflow; zero when water is
    conserved.  The flow volumes of neighbouring cells cancel in the sum."""
    return abs(float(np.sum(m)))


def test_config2_plain_prefix():
    """The plain FP64 path on the 256x256x64 block, first four accepted steps: same time
    steps, same Newton and Krylov counts, heads within 1e-8, step volumes within 1e-10 of
    the inflow."""
    from msg123_b200.solver import GpuSolver
    p = make_config("hetero")
    g, o = GpuSolver(p, **PLAIN), Oracle(p, **PLAIN)
    g.init_state(); o.init_state()
    for k in range(4):
        rg, sg = g.advance(nsteps=1)
        ro, so = o.advance(nsteps=1)
        print(f"step {k + 1}: gpu newton {sg['newton_total']} krylov {sg['krylov_total']} t {sg['current_t']}; "
              f"oracle newton {so['newton_total']} krylov {so['krylov_total']} t {so['current_t']}")
        assert rg == ro == 0
        assert sg["current_t"] == so["current_t"]
        assert sg["newton_total"] == so["newton_total"] and sg["krylov_total"] == so["krylov_total"]
    hg, ho = g.get_state()["head_new"], o.get_state()["head_new"]
    err = relmax(hg, ho)
    mg, mo = g.calc_mass(), o.calc_mass()
    inflow = abs(mo[2])
    print(f"config 2 prefix: head rel {err:.2e}, mass {np.max(np.abs(mg - mo)) / inflow:.2e} of inflow")
    assert err <= HEAD_TOL
    assert np.max(np.abs(mg - mo)) <= 1e-10 * inflow
    g.close(); o.close()


def test_value_path_against_tight_fp64():
    """The benchmark's value path against the FP64 oracle solved to criteria 1e-11: heads
    within 1e-8 after 8 and after 12 steps (measured 1.6e-9 and 2.8e-9); every step's
    volumes within 1e-10 of the step's inflow of the oracle's (measured <= 4e-12), and the
    GPU run's own mass balance closing to 1e-10 of the inflow (measured <= 4e-12)."""
    from msg123_b200.learned import Cnn
    from msg123_b200.solver import GpuSolver
    from msg123_b200.train_guess import load
    p = make_config("large", shape=(128, 128, 64))
    sched = dict(sim_type=0, inc_fact=1.1, ini_step=600.0)
    g = GpuSolver(p, **VALUE, **sched)
    cnn = load(Cnn(seed=0))
    cnn.attach(g)
    o = Oracle(p, precon_type=1, ref_quirks=0, precision=0, amg_lag=1, guess_mode=1, vg_form=0,
               criteria=1e-11, maxout_iter=60, **sched)
    g.init_state(); o.init_state()
    worst_closure, worst_vol = 0.0, 0.0
    for k in range(12):
        rg, sg = g.advance(nsteps=1)
        mg = g.calc_mass()
        ro, so = o.advance(nsteps=1)
        mo = o.calc_mass()
        assert rg == ro == 0 and sg["accepted"] == so["accepted"] == 1
        assert sg["current_t"] == so["current_t"]
        inflow = abs(mo[2]) + abs(mo[7])
        worst_closure = max(worst_closure, closure(mg) / inflow)
        worst_vol = max(worst_vol, float(np.max(np.abs(mg - mo))) / inflow)
        line = (f"step {k + 1} t {sg['current_t']:.0f}: gpu newton {sg['newton_total']} krylov {sg['krylov_total']}; "
                f"oracle(1e-11) newton {so['newton_total']}; closure gpu {closure(mg) / inflow:.1e} "
                f"oracle {closure(mo) / inflow:.1e}; volumes gpu-oracle {np.max(np.abs(mg - mo)) / inflow:.1e}")
        if k in (7, 11):
            err = relmax(g.get_state()["head_new"], o.get_state()["head_new"])
            line += f"; head rel {err:.2e}"
            assert err <= HEAD_TOL, (k + 1, err)
        print(line)
    print("fallbacks", g.guess_fallbacks(), "worst closure", worst_closure, "worst volume difference", worst_vol)
    assert worst_closure <= 1e-10 and worst_vol <= 1e-10
    g.close(); o.close(); cnn.close()


def test_reference_amg_mode_run():
    """precon_type = 1 with ref_quirks = 1 -- what a deck with the reference's AMG setting
    runs -- over six adaptive steps: identical time steps and counts, heads within 1e-8."""
    from msg123_b200.solver import GpuSolver
    p = make_config("hetero", shape=(48, 40, 16), seed=9)
    kw = dict(precon_type=1, ref_quirks=1, precision=0, amg_lag=0, guess_mode=0, vg_form=0)
    g, o = GpuSolver(p, **kw), Oracle(p, **kw)
    g.init_state(); o.init_state()
    rg, sg = g.advance(nsteps=6)
    ro, so = o.advance(nsteps=6)
    print("reference AMG mode: gpu", sg, "oracle", so)
    assert rg == ro == 0
    assert sg["current_t"] == so["current_t"] and sg["rejected"] == so["rejected"]
    assert sg["newton_total"] == so["newton_total"] and sg["krylov_total"] == so["krylov_total"]
    assert sg["back_total"] == so["back_total"]
    assert relmax(g.get_state()["head_new"], o.get_state()["head_new"]) <= HEAD_TOL
    mg, mo = g.calc_mass(), o.calc_mass()
    assert np.max(np.abs(mg - mo)) <= 1e-10 * abs(mo[2])
    g.close(); o.close()


def test_ensemble_members_against_oracle():
    """Three members advanced together by the batched driver (mixed precision, AMG kept for
    4 steps, extrapolated guess), each against the FP64 oracle solved to criteria 1e-10 on
    the member's own field at the same times: heads within 1e-8.  The members are small
    ones (for the oracle's time) whose tight-tolerance oracle run takes the same time steps:
    member 31 (sigma_lnK 1.38) rejects its second step even at 60 Newton iterations with
    criteria 1e-10, so no same-time comparison exists for it."""
    from msg123_b200.ensemble import Ensemble, ENSEMBLE
    seeds = [20, 29, 35]                        # 219k, 209k and 230k cells
    # the first step from the hydrostatic start takes more than the default 20 Newton
    # iterations at criteria 1e-10; both sides get the same cap, so no step is rejected
    sched = dict(sim_type=0, inc_fact=1.1, ini_step=600.0, maxout_iter=60)
    ens = Ensemble(seeds=seeds, **sched)
    ens.init_state()
    dt, stats = ens.advance(4, workers=3)
    assert all(s["status"] == 0 and s["accepted"] == 4 and s["rejected"] == 0 for s in stats)
    for k, seed in enumerate(seeds):
        p = make_member(seed, **sched)
        o = Oracle(p, **dict(ENSEMBLE, precision=0, amg_lag=1, criteria=1e-10))
        o.init_state()
        ro, so = o.advance(nsteps=4)
        assert ro == 0 and so["current_t"] == stats[k]["current_t"]
        err = relmax(ens.members[k].get_state()["head_new"], o.get_state()["head_new"])
        print(f"member {seed} ({p.nx}x{p.ny}x{p.nz}): gpu newton {stats[k]['newton_total']}, "
              f"oracle(1e-10) newton {so['newton_total']}, head rel {err:.2e}")
        assert err <= HEAD_TOL
        o.close()
    ens.close()
