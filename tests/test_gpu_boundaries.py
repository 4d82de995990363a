"""Wells, rivers and lakes on the GPU against the oracle.

A river over three top cells, a lake over one and two three-cell wells (one extracting,
one injecting) on a heterogeneous block: calc_func and make_matvec on the same state
(residual within 1e-12 of max|F|, Jacobian diagonal within 1e-6 relative like the other
assembly tests), then three adaptive time steps with the well rates set at each step
(heads within 1e-8, the nine step volumes within 1e-10 of the inflow volume, the per-cell
well, river and lake volumes within 1e-12 of their largest).
"""
import numpy as np
import pytest

from msg123_b200.config import make_config
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def tables(p):
    nx, ny, S = p.nx, p.ny, p.ncals
    top = p.cell_top[:S]
    rc = np.array([2, nx + 3, 2 * nx + 4])
    riv = (rc, top[rc - 1] + 0.02, top[rc - 1] - 0.05, np.full(3, 2.5))
    lc = np.array([S - 1])
    lak = (lc, top[lc - 1] - 0.01, top[lc - 1] - 0.2, np.array([1.7]))
    c1, c2 = 1 + nx // 2 + nx * (ny // 2), 2 + nx
    col = lambda c: np.array([c + k * S for k in (1, 2, 3)])
    bott = float(p.cell_top[-1]) - 1.0
    wells = (np.array([0, 3, 6]), np.concatenate([col(c1), col(c2)]), np.full(6, 0.8), np.array([bott, bott]),
             np.array([-2.0e-4, 1.0e-4]))
    return riv, lak, wells


def setup(p):
    from msg123_b200.solver import GpuSolver
    g, o = GpuSolver(p), Oracle(p)
    riv, lak, wells = tables(p)
    for s in (g, o):
        s.set_rivers(*riv)
        s.set_lakes(*lak)
        s.set_wells(*wells)
    return g, o


def test_boundary_terms_residual_and_jacobian():
    p = make_config("hetero", shape=(20, 16, 10), seed=5)
    g, o = setup(p)
    g.init_state(); o.init_state()
    h = p.cell_top + np.random.default_rng(3).uniform(-0.3, 0.05, p.ncalc)
    for s in (g, o):
        s.set_state(head_new=h, delt=600.0)
    fg, fo = g.calc_func(h), o.calc_func(h)
    assert np.max(np.abs(fg - fo)) <= 1e-12 * np.max(np.abs(fo))
    dg, lug, rg = g.make_matvec()
    do, luo, ro = o.make_matvec()
    assert np.max(np.abs(rg - ro)) <= 1e-12 * np.max(np.abs(ro))
    assert np.max(np.abs(dg - do) / np.maximum(np.abs(do), 1e-300)) <= 1e-6
    g.close(); o.close()


def test_boundary_terms_over_steps():
    p = make_config("hetero", shape=(20, 16, 10), seed=5)
    g, o = setup(p)
    g.init_state(); o.init_state()
    rg, sg = g.advance(nsteps=3)
    ro, so = o.advance(nsteps=3)
    print("gpu", sg, "oracle", so)
    assert rg == ro == 0 and sg["current_t"] == so["current_t"]
    hg, ho = g.get_state()["head_new"], o.get_state()["head_new"]
    assert np.max(np.abs(hg - ho)) / np.max(np.abs(ho)) <= 1e-8
    mg, mo = g.calc_mass(), o.calc_mass()
    inflow = abs(mo[2]) + abs(mo[3]) + abs(mo[5]) + abs(mo[6])
    assert mo[3] != 0 and mo[5] != 0 and mo[6] != 0
    assert np.max(np.abs(mg - mo)) <= 1e-10 * inflow
    st = g.get_state()
    o.set_state(head_new=st["head_new"], head_old=st["head_old"], srat_old=st["srat_old"],
                surf_head=st["surf_head"], delt=sg["delt"])
    cg, co = g.cell_mass(), o.cell_mass()
    for k in ("wel", "riv", "lak"):
        scale = np.max(np.abs(co[k]))
        assert scale > 0 and np.max(np.abs(cg[k] - co[k])) <= 1e-12 * scale, k
    g.close(); o.close()


def test_boundary_tables_rejected():
    """Tables the reference could not run deterministically are refused before any device
    work: a cell in two wells, a surface cell listed twice, cells out of range."""
    from msg123_b200.solver import GpuSolver, MsgError
    p = make_config("hetero", shape=(6, 5, 4), seed=1)
    g = GpuSolver(p)
    with pytest.raises(MsgError):
        g.set_wells([0, 1, 2], [7, 7], [1.0, 1.0], [0.0, 0.0], [1e-4, 1e-4])
    with pytest.raises(MsgError):
        g.set_rivers([3, 3], [1.0, 1.0], [0.0, 0.0], [1.0, 1.0])
    with pytest.raises(MsgError):
        g.set_lakes([31], [1.0], [0.0], [1.0])
    with pytest.raises(MsgError):
        g.set_wells([0, 1], [p.ncalc + 1], [1.0], [0.0], [1e-4])
    g.set_wells([0], [], [], [], [])                     # no wells: allowed, clears the table
    g.close()
