"""AMG on the GPU against the CPU oracle's restatement of the same algorithm.

The setup (strength filter, MIS-2 aggregation, smoothed prolongation, R = P^T and
the Galerkin product) is deterministic and fixes every summation order, so the
hierarchy must match the oracle bit for bit; so must one V-cycle.
"""
import numpy as np
import pytest

from msg123_b200.config import make_config
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

AMG = dict(precon_type=1, ref_quirks=0, amg_coarse_max=200)


def system(shape=(24, 20, 16), seed=6, delt=3600.0, **kw):
    p = make_config("hetero", shape=shape, seed=seed, **kw)
    o = Oracle(p, **AMG)
    o.init_state()
    o.set_state(head_new=p.head0 + 0.004 * np.random.default_rng(seed).standard_normal(p.ncalc), delt=delt)
    d, lu, r = o.make_matvec()
    return p, o, d, lu, r


# Run tests use 600-s steps.  With 1800-s steps from the dry hydrostatic start of these
# 32x28x16 blocks the first steps meet the seepage switch (the surface term is not
# differentiable where h = surf_top) and Newton with the reference's step-size test can
# stagnate in the line search: on the seed-14 block the oracle's own runs at criteria
# 1e-10 and 1e-12 end 1.8e-8 apart, so no run there pins 1e-8.  At 600 s the criteria-1e-8
# run lies within 2e-9 of the criteria-1e-12 run (seeds 12 and 14).


def check_heads(p, ov, steps, hg, ho, sg, so):
    """Heads of a GPU run (hg) and an oracle run (ho) of the same method and time steps.
    When both take the same Newton iterations they follow the same path up to rounding and
    must agree to 1e-8 (measured ~1e-14).  The GPU's dot products are summed in a fixed tree
    order rather than the oracle's serial order, and that can flip one stopping decision;
    the two runs then stop at different points, each as far from the converged answer as
    the stopping rule allows (|dh| <= 1e-8 max|h| on a linearly converging iteration leaves
    up to ~3e-8, for both implementations alike).  Such a pair is run again at criteria
    1e-10 on both sides, where the two converge to the same heads within 1e-8."""
    rel = lambda a, b: float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    if sg["newton_total"] == so["newton_total"]:
        assert rel(hg, ho) <= 1e-8
        return rel(hg, ho)
    from msg123_b200.solver import GpuSolver
    tight = dict(ov, criteria=1e-10, maxout_iter=60)
    g, t = GpuSolver(p, **tight), Oracle(p, **tight)
    g.init_state(); t.init_state()
    rg, sgt = g.advance(nsteps=steps)
    rt, stt = t.advance(nsteps=steps)
    # the tight pair may take other time steps than the criteria-1e-8 pair (a step the
    # looser run rejected at 20 iterations converges within 60), but the same as each other
    assert rg == rt == 0 and sgt["current_t"] == stt["current_t"]
    hgt, ht = g.get_state()["head_new"], t.get_state()["head_new"]
    same_t = sgt["current_t"] == sg["current_t"]
    print("Newton counts differ at criteria 1e-8: gpu", sg["newton_total"], "oracle", so["newton_total"],
          "(gpu vs oracle", rel(hg, ho), ") -> at criteria 1e-10: gpu vs oracle", rel(hgt, ht),
          *(("; the criteria-1e-8 runs from it: gpu", rel(hg, ht), "oracle", rel(ho, ht)) if same_t else ()))
    assert rel(hgt, ht) <= 1e-8
    g.close(); t.close()
    return rel(hgt, ht)


def gpu(p, **kw):
    from msg123_b200.solver import GpuSolver
    prm = dict(AMG)
    prm.update(kw)
    return GpuSolver(p, **prm)


@pytest.mark.parametrize("shape,seed", [((24, 20, 16), 6), ((40, 36, 20), 8), ((9, 7, 5), 1)])
def test_hierarchy_bitexact(shape, seed):
    p, o, d, lu, r = system(shape, seed)
    o.set_system(d, lu, r)
    g = gpu(p)
    g.set_system(d, lu, r)
    lo, lg = o.amg_levels(), g.amg_levels()
    assert len(lo) == len(lg) and len(lo) >= 2
    for k in range(1, len(lo)):
        a, b = lg[k], lo[k]
        assert a["n"] == b["n"], k
        for key in ("agg", "pindex", "poffrow", "offind", "offrow"):
            assert np.array_equal(a[key], b[key]), (k, key)
        for key in ("pval", "dmat", "lumat"):
            assert np.array_equal(a[key], b[key]), (k, key)


def test_vcycle_bitexact():
    p, o, d, lu, r = system((32, 28, 18), 3)
    o.set_system(d, lu, r)
    g = gpu(p)
    g.set_system(d, lu, r)
    v = np.random.default_rng(5).standard_normal(p.ncalc)
    zg, zo = g.precond(v), o.precond(v)
    assert np.array_equal(zg, zo)


def test_amg_bicgstab_counts():
    p, o, d, lu, r = system((32, 28, 18), 3)
    o2 = Oracle(p, maxinn_iter=100, **AMG)
    o2.set_system(d, lu, r)
    g = gpu(p, maxinn_iter=100)
    g.set_system(d, lu, r)
    b2 = float(r @ r)
    xg, _, itg, cg = g.solve_linalg(b2, 1e-10)
    xo, _, ito, co = o2.solve_linalg(b2, 1e-10)
    assert itg == ito and cg == co == 1
    assert np.max(np.abs(xg - xo)) <= 1e-9 * np.max(np.abs(xo))


def test_amg_run_parity():
    p = make_config("hetero", shape=(32, 28, 16), seed=12)
    ov = dict(AMG, sim_type=0, inc_fact=1.0, ini_step=600.0)
    from msg123_b200.solver import GpuSolver
    g, o = GpuSolver(p, **ov), Oracle(p, **ov)
    g.init_state(); o.init_state()
    rg, sg = g.advance(nsteps=3)
    ro, so = o.advance(nsteps=3)
    assert rg == ro == 0
    hg, ho = g.get_state()["head_new"], o.get_state()["head_new"]
    check_heads(p, ov, 3, hg, ho, sg, so)
    mg, mo = g.calc_mass(), o.calc_mass()
    assert np.max(np.abs(mg - mo)) <= 1e-10 * abs(mo[2])
    print("GPU", sg, "CPU", so)


@pytest.mark.parametrize("n,seed", [(1, 0), (7, 1), (128, 2), (300, 3)])
def test_dense_inverse_bitexact(n, seed):
    from msg123_b200.solver import dense_inverse as gpu_inv
    from oracle.oracle import dense_inverse as cpu_inv
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + n * np.eye(n) * rng.uniform(0.5, 2.0)
    ig, io = gpu_inv(a), cpu_inv(a)
    assert np.array_equal(ig, io)
    assert np.allclose(ig @ a, np.eye(n), atol=1e-10)


def test_amg_lagged_setup_parity():
    """amg_lag = 1 (hierarchy of the first Newton iteration kept for the time step)."""
    p = make_config("hetero", shape=(32, 28, 16), seed=13)
    ov = dict(AMG, amg_lag=1, sim_type=0, inc_fact=1.0, ini_step=600.0)
    from msg123_b200.solver import GpuSolver
    g, o = GpuSolver(p, **ov), Oracle(p, **ov)
    g.init_state(); o.init_state()
    rg, sg = g.advance(nsteps=3)
    ro, so = o.advance(nsteps=3)
    assert rg == ro == 0
    hg, ho = g.get_state()["head_new"], o.get_state()["head_new"]
    check_heads(p, ov, 3, hg, ho, sg, so)


def test_amg_lag_over_steps_parity():
    """amg_lag = 3: one hierarchy serves three time steps; same rule in the oracle."""
    p = make_config("hetero", shape=(32, 28, 16), seed=14)
    ov = dict(AMG, amg_lag=3, sim_type=0, inc_fact=1.0, ini_step=600.0)
    from msg123_b200.solver import GpuSolver
    g, o = GpuSolver(p, **ov), Oracle(p, **ov)
    g.init_state(); o.init_state()
    rg, sg = g.advance(nsteps=5)
    ro, so = o.advance(nsteps=5)
    assert rg == ro == 0
    hg, ho = g.get_state()["head_new"], o.get_state()["head_new"]
    err = check_heads(p, ov, 5, hg, ho, sg, so)
    print("newton GPU", sg["newton_total"], "oracle", so["newton_total"], "head err", err)


def test_jv_mode_run_parity():
    """jv_mode = 1 (the line-search slope from BiCGStab's own residual, J dh = rhs - r):
    GPU and oracle implement it alike, so the runs match as the FP64 AMG runs do, and they
    land within 1e-8 of the jv_mode = 0 run (the slope changes the line search only)."""
    p = make_config("hetero", shape=(32, 28, 16), seed=12)
    ov = dict(AMG, sim_type=0, inc_fact=1.0, ini_step=600.0, amg_lag=1, jv_mode=1)
    from msg123_b200.solver import GpuSolver
    g, o = GpuSolver(p, **ov), Oracle(p, **ov)
    g.init_state(); o.init_state()
    rg, sg = g.advance(nsteps=3)
    ro, so = o.advance(nsteps=3)
    assert rg == ro == 0
    hg, ho = g.get_state()["head_new"], o.get_state()["head_new"]
    err = check_heads(p, ov, 3, hg, ho, sg, so)
    g0 = GpuSolver(p, **dict(ov, jv_mode=0))
    g0.init_state()
    r0, s0 = g0.advance(nsteps=3)
    h0 = g0.get_state()["head_new"]
    print("jv_mode 1: newton", sg["newton_total"], "jv_mode 0:", s0["newton_total"], "err vs oracle", err,
          "vs jv_mode 0", np.max(np.abs(hg - h0)) / np.max(np.abs(h0)))
    assert r0 == 0 and np.max(np.abs(hg - h0)) / np.max(np.abs(h0)) <= 1e-8
