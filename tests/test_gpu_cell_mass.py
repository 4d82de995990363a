"""Per-cell mass-balance volumes (calc_cell_mas, Calc_output.f90:54-91) on the GPU
against the oracle, on the same state.

Both sides are given the same time levels (the GPU's state after a few steps is copied
into the oracle), so the comparison isolates the volume arithmetic: every per-cell array
within 1e-11 of its largest entry (the storage change subtracts two saturations, which
turns last-bit pow differences into ~2e-12 of the largest volume), and the per-cell arrays of the GPU summing to its
whole-grid totals (msg_gpu_calc_mass) within 1e-10 of the inflow volume.
"""
import numpy as np
import pytest

from msg123_b200.config import make_config
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

CASES = [
    ("box", dict(shape=(12, 10, 16)), {}),                 # sea layer on top, free drainage
    ("hetero", dict(shape=(24, 20, 12), seed=4), {}),      # recharge, surface term
]


@pytest.mark.parametrize("name,kw,ov", CASES, ids=[c[0] for c in CASES])
def test_cell_mass_matches_oracle(name, kw, ov):
    from msg123_b200.solver import GpuSolver
    p = make_config(name, **kw)
    g, o = GpuSolver(p, **ov), Oracle(p, **ov)
    g.init_state(); o.init_state()
    rg, sg = g.advance(nsteps=3)
    ro, so = o.advance(nsteps=3)
    assert rg == ro == 0
    st = g.get_state()
    o.set_state(head_new=st["head_new"], head_old=st["head_old"], srat_old=st["srat_old"],
                surf_head=st["surf_head"], delt=sg["delt"])
    cg, co = g.cell_mass(), o.cell_mass()
    for k in ("sto", "con", "sea", "rec", "sur", "drn"):
        scale = max(np.max(np.abs(co[k])), 1e-300)
        err = np.max(np.abs(cg[k] - co[k])) / scale
        assert err <= 1e-11, (k, err)
    for k in ("wel", "riv", "lak"):
        assert not np.any(cg[k])
    tot = g.calc_mass()
    sums = [cg["sto"].sum(), cg["con"].sum(), cg["rec"].sum(), 0.0, cg["sur"].sum(), 0.0, 0.0, cg["sea"].sum(),
            cg["drn"].sum()]
    inflow = abs(tot[2]) + abs(tot[7])
    assert inflow > 0
    assert np.max(np.abs(np.array(sums) - tot)) <= 1e-10 * inflow
    g.close(); o.close()
