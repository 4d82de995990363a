"""The synthetic input generator (msg123_b200/config.py): seeded and repeatable, soil
parameters quantised to real(SP) as the reference reads them (Assign_calculation.f90:19-21),
len_scal = 10^ceil(log10 max|z|) (Read_input.f90:1100-1112), and the hydrostatic start of
the heterogeneous block at rest (F = 0 before any rain)."""
import numpy as np
import pytest

from msg123_b200.config import len_scale, make_config


@pytest.mark.parametrize("name,kw", [("box", dict(shape=(4, 3, 5))), ("hetero", dict(shape=(8, 6, 4), seed=3)),
                                     ("box1r", dict(shape=(4, 3, 5)))])
def test_generator_is_seeded_and_single_precision(name, kw):
    a, b = make_config(name, **kw), make_config(name, **kw)
    for f in ("reta", "retn", "resi", "poro", "ss", "ksx", "ksy", "ksz", "cell_top", "head0", "rech"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    for f in ("reta", "retn", "resi", "poro", "ss", "ksx", "ksy", "ksz"):
        assert getattr(a, f).dtype == np.float32, f
    assert a.ncalc == int(np.prod(kw["shape"])) and a.ncals == kw["shape"][0] * kw["shape"][1]


def test_other_seed_other_field():
    a, b = make_config("hetero", shape=(8, 6, 4), seed=3), make_config("hetero", shape=(8, 6, 4), seed=4)
    assert not np.array_equal(a.ksz, b.ksz)


@pytest.mark.parametrize("zmax,ls", [(0.2, 1.0), (1.0, 1.0), (1.1, 10.0), (10.0, 10.0), (16.0, 100.0), (250.0, 1000.0)])
def test_len_scale(zmax, ls):
    assert float(len_scale(zmax)) == ls


def test_hydrostatic_start_is_at_rest():
    from oracle.oracle import Oracle
    p = make_config("hetero", shape=(8, 6, 4), seed=3)
    o = Oracle(p)
    o.init_state()
    o.set_recharge(np.zeros(p.ncals))
    assert np.max(np.abs(o.calc_func(p.head0))) <= 1e-20
