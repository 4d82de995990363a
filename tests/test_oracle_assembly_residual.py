"""The identity behind the assembly ahead of the line search: the right-hand side that
make_matvec assembles at a head (Make_linearsystem.f90:24-68, rhs = -F) is, bit for bit,
minus the residual calc_func evaluates at the same head (Calc_function.f90:24-101) -- the
assembly forms every term of F with the same operations in the same order -- so the sum of
squares, and every decision taken from it, is the same too.  Checked in the oracle on the
boundary mixes it supports: rain on a heterogeneous block, a sea-layer top with a no-flow
bottom, a ponded top with free drainage, and wells, a river and a lake, in both van
Genuchten forms."""
import numpy as np
import pytest

from msg123_b200.config import make_config
from oracle.oracle import Oracle


def _stages(p):
    nx, S = p.nx, p.ncals
    top = p.cell_top[:S]
    rc = np.array([2, nx + 3])
    riv = (rc, top[rc - 1] + 0.02, top[rc - 1] - 0.05, np.full(2, 2.5))
    lc = np.array([S - 1])
    lak = (lc, top[lc - 1] - 0.01, top[lc - 1] - 0.2, np.array([1.7]))
    c1 = 1 + nx // 2
    bott = float(p.cell_top[-1]) - 1.0
    wells = (np.array([0, 2]), np.array([c1 + S, c1 + 2 * S]), np.full(2, 0.8), np.array([bott]),
             np.array([-1.0e-4]))
    return riv, lak, wells


@pytest.mark.parametrize("vg_form", [0, 1])
@pytest.mark.parametrize("name,kw,boundaries", [("hetero", dict(shape=(12, 10, 8), seed=3), False),
                                                ("hetero", dict(shape=(10, 9, 6), seed=7), True),
                                                ("box1r", dict(shape=(6, 5, 7)), False),
                                                ("box", dict(shape=(6, 5, 7)), False)])
def test_assembled_rhs_is_minus_residual(name, kw, boundaries, vg_form):
    p = make_config(name, **kw)
    o = Oracle(p, vg_form=vg_form)
    if boundaries:
        riv, lak, wells = _stages(p)
        o.set_rivers(*riv)
        o.set_lakes(*lak)
        o.set_wells(*wells)
    o.init_state()
    h = p.head0 + 0.003 * np.random.default_rng(1).standard_normal(p.ncalc)
    o.set_state(head_new=h, delt=1800.0)
    _, _, rhs = o.make_matvec()
    f = o.calc_func(h)
    assert np.array_equal(rhs, -f)
    assert float(np.sum(f * f)) == float(np.sum(rhs * rhs))
    o.close()
