"""Output series in the reference's binary format and the water table behind one of them.

CPU: the record layout of write_header_bin + write_3dbin / write_2dbin (Write_module.f90:
61-99,146-225) -- float32 time, then float32(value * unit) x fastest -- written and read
back; the water-table restatement (calc_wtable, Calc_output.f90:20-52) on hand-made
columns.  GPU: the device water table equals the restatement on a solved state, and the
three series written from that state read back as the reference would have written them.
"""
import numpy as np
import pytest

from msg123_b200 import refout
from oracle.output_ref import water_table


def test_record_layout_and_round_trip(tmp_path):
    nx, ny, nz = 3, 2, 4
    rng = np.random.default_rng(0)
    h1, h2 = rng.standard_normal(nx * ny * nz), rng.standard_normal(nx * ny * nz)
    unit = np.float32(10.0)
    p = tmp_path / "head.bin"
    refout.append(p, 1800.0, h1, unit, (nx, ny, nz))
    refout.append(p, 3600.0, h2, unit, (nx, ny, nz))
    raw = np.fromfile(p, dtype="<f4")
    assert raw.size == 2 * (1 + nx * ny * nz)
    assert raw[0] == np.float32(1800.0)
    # cell (x=2, y=1, z=1) is the second value; (x=1, y=2, z=1) the fourth; (1, 1, 2) the seventh
    assert raw[1 + 1] == np.float32(h1[1] * 10.0)
    assert raw[1 + 3] == np.float32(h1[3] * 10.0)
    assert raw[1 + 6] == np.float32(h1[6] * 10.0)
    recs = refout.read(p, (nx, ny, nz))
    assert [t for t, _ in recs] == [1800.0, 3600.0]
    assert recs[1][1].shape == (nz, ny, nx)
    assert np.array_equal(recs[1][1].reshape(-1), (h2 * np.float64(unit)).astype(np.float32))
    w = tmp_path / "wtab.bin"
    refout.append(w, 5.0, h1[: nx * ny], 1.0, (nx, ny))
    (t, a), = refout.read(w, (nx, ny))
    assert t == 5.0 and a.shape == (ny, nx) and np.array_equal(a.reshape(-1), h1[: nx * ny].astype(np.float32))
    with pytest.raises(ValueError):
        refout.read(p, (nx, ny, nz + 1))
    with pytest.raises(ValueError):
        refout.append(p, 0.0, h1[:-1], 1.0, (nx, ny, nz))


def test_product_rounds_once():
    """real(value * unit, SP): the product in double, one rounding to single."""
    v = np.array([0.1234567890123, -3.333333333333])
    unit = 100.0
    assert np.array_equal(refout.field(v, unit, (2, 1)), (v * 100.0).astype(np.float32))


def test_water_table_restatement_by_hand():
    nx, ny, nz = 3, 1, 4
    # columns: 0 fully saturated, 1 unsaturated at the bottom, 2 saturated below layer 1
    srat = np.array([[1.0, 0.9, 0.8],
                     [1.0, 0.9, 0.7],
                     [1.0, 0.95, 1.0],
                     [1.0, 0.99, 1.0]])
    head = np.arange(12, dtype=np.float64).reshape(nz, nx * ny) + 0.5
    wt = water_table(head.reshape(-1), srat.reshape(-1), nx, ny, nz)
    assert wt[0] == head[0, 0]      # whole column saturated: top cell
    assert wt[1] == head[3, 1]      # bottom cell already unsaturated
    assert wt[2] == head[1, 2]      # lowest unsaturated cell above the saturated ones


@pytest.mark.gpu
def test_gpu_water_table_and_series(tmp_path):
    from msg123_b200.config import make_config
    from msg123_b200.solver import GpuSolver
    p = make_config("hetero", shape=(24, 20, 16), seed=9)
    g = GpuSolver(p, precision=1, amg_lag=4)
    g.init_state()
    rc, st = g.advance(nsteps=4)
    assert rc == 0
    s = g.get_state()
    wt = g.water_table()
    ref = water_table(s["head_new"], s["srat_new"], p.nx, p.ny, p.nz)
    assert np.array_equal(wt, ref)
    # the hydrostatic start puts the water table inside the block: some columns must pass
    # saturated cells on the way up
    assert np.any(s["srat_new"] == 1.0) and np.any(s["srat_new"] < 1.0)
    ls = p.params["len_scal"]
    prefix = str(tmp_path / "run")
    refout.write_state(prefix, g, st["current_t"], ls)
    (t, h), = refout.read(prefix + "_head.bin", (p.nx, p.ny, p.nz))
    assert t == np.float32(st["current_t"])
    assert np.array_equal(h.reshape(-1), (s["head_new"] * np.float64(np.float32(ls))).astype(np.float32))
    (_, sr), = refout.read(prefix + "_srat.bin", (p.nx, p.ny, p.nz))
    assert np.array_equal(sr.reshape(-1), s["srat_new"].astype(np.float32))
    (_, w), = refout.read(prefix + "_wtab.bin", (p.nx, p.ny))
    assert np.array_equal(w.reshape(-1), (ref * np.float64(np.float32(ls))).astype(np.float32))


def test_input_field_round_trip(tmp_path):
    nx, ny, nz = 4, 3, 2
    v = np.random.default_rng(1).standard_normal(nx * ny * nz).astype(np.float32)
    p = tmp_path / "ks.bin"
    refout.write_field(p, v, (nx, ny, nz))
    assert p.stat().st_size == 4 * nx * ny * nz
    a = refout.read_field(p, (nx, ny, nz))
    assert a.shape == (nz, ny, nx) and a[1, 0, 2] == v[nx * ny + 2]
    with pytest.raises(ValueError):
        refout.read_field(p, (nx, ny))


@pytest.mark.parametrize("x,expect", [
    (123.456, " 0.123456E+03"), (-0.001234567, "-0.123457E-02"), (0.0, " 0.000000E+00"),
    (9.9999996, " 0.100000E+02"), (1e100, " 0.100000+101"), (-1e-120, "-0.100000-119"),
])
def test_ew_edit_descriptor(x, expect):
    assert refout.ew(x) == expect


def test_mass_balance_file(tmp_path):
    p = tmp_path / "mass.csv"
    ls = 10.0
    mb = refout.MassBalance(p, "SEC", ls)
    step = [-1.0e-3, 2.0e-3, 5.0e-4, 0.0, -1.0e-4, 0.0, 0.0, 3.0e-4, -1.5e-4]   # sto, flow, rech, ..., drain
    mb.add_step(step)
    mb.add_step(step)
    line = mb.write(3600.0)
    lines = p.read_text().splitlines()
    assert lines[0] == "SEC,whole area"
    assert lines[1] == ",FLOW,STORAGE,RECHARGE,WELL,SURFACE,RIVER,LAKE,SEA,ALL"
    assert lines[2] == line and line.count(",") == 9 and all(len(t) == 13 for t in line.split(","))
    (row,) = refout.read_mass(p)
    c = 1000.0                                         # len_scal**3
    assert row["time"] == 3600.0
    assert row["FLOW"] == pytest.approx(2 * 2.0e-3 * c, rel=1e-6)
    assert row["STORAGE"] == pytest.approx(2 * -1.0e-3 * c, rel=1e-6)
    assert row["SEA"] == pytest.approx(2 * 3.0e-4 * c, rel=1e-6)
    assert row["ALL"] == pytest.approx(2 * sum(step) * c, rel=1e-6)
    mb.add_step(step)
    mb.write(7200.0)                                   # the sums restart after each output
    rows = refout.read_mass(p)
    assert len(rows) == 2 and rows[1]["FLOW"] == pytest.approx(2.0e-3 * c, rel=1e-6)
