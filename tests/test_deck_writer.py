"""Reference-format deck writer and reader (msg123_b200/deck.py: write_deck, read_deck).

A generated problem is written as msg123.main plus the files it names (type-7 grid,
retention / parameter compile files with 3D float32 fields, 3D float64 initial heads, the
time-series file with rain records and a sea level, a region file for a ponded top), read
back the way the reference reads and scales it, and compared with the generator's arrays:
soil parameters bit for bit, elevations and heads to the rounding of the reference's
real(SP) / real(DP) products.  The oracle then runs both problems with the same settings.
No Fortran build exists here, so the deck itself is checked against the reader in this file
and against the namelist and record layouts the reference's readers use."""
import os

import numpy as np
import pytest

from msg123_b200.config import make_config
from msg123_b200.deck import read_deck, read_namelists, write_deck, SNOVAL
from oracle.oracle import Oracle

FIELDS = ("reta", "retn", "resi", "poro", "ss", "ksx", "ksy", "ksz")
GEOM = ("cell_top", "cell_vol", "dis2face", "face_area", "area_r", "surf_top", "surf_bott")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(a)), 1e-300))


@pytest.mark.parametrize("name,kw,geom_tol", [("hetero", dict(shape=(8, 6, 4)), 0.0),
                                              ("box1r", dict(shape=(4, 4, 5)), 1e-6)])
def test_roundtrip(tmp_path, name, kw, geom_tol):
    p = make_config(name, **kw)
    files = write_deck(p, str(tmp_path))
    assert "msg123.main" in files and all(os.path.exists(tmp_path / f) for f in files)
    q = read_deck(str(tmp_path))
    assert (q.nx, q.ny, q.nz, q.sea_top, q.free_drainage) == (p.nx, p.ny, p.nz, p.sea_top, 0)
    for k in FIELDS:
        assert np.array_equal(getattr(q, k), getattr(p, k)), k
    for k in GEOM:
        assert rel(getattr(p, k), getattr(q, k)) <= geom_tol, k
    assert rel(p.head0, q.head0) <= 1e-8
    assert np.array_equal(q.rech, p.rech) and np.array_equal(q.sea_head, p.sea_head)
    assert q.rech_until == p.rech_until
    assert q.params["len_scal"] == p.params["len_scal"]
    for k in ("maxout_iter", "maxinn_iter", "precon_type", "ini_step", "max_step", "inc_fact", "sim_type"):
        assert q.params[k] == pytest.approx(p.params[k]), k


def test_layouts(tmp_path):
    """The files follow the layouts the reference's readers take: namelist groups in the
    order read_main_file reads them (Read_input.f90:23-61); float32 streams of nx*ny*nz
    values for the fields (Read_module.f90:459-485); float64 initial heads; rain records of
    one float32 end time (hours) and nx*ny float32 values (mm/h); the sea level -9999 outside
    the sea layer; the region file -1 / 0 / 1 by layer."""
    p = make_config("box1r", shape=(4, 4, 5))
    write_deck(p, str(tmp_path))
    order = [l.strip()[1:].lower() for l in open(tmp_path / "msg123.main") if l.startswith("&")]
    assert order == ["set_simulation", "set_calc_time", "set_calc_reg", "set_solution", "set_grid",
                     "set_retn_parm", "set_init", "set_time_input", "set_geog", "set_wtab", "set_mass",
                     "set_out_vari", "set_out_unit", "set_out_time"]
    nxy, nzd = 16, 7
    assert np.fromfile(tmp_path / "alpha.bin", dtype="<f4").size == nxy * nzd
    assert np.fromfile(tmp_path / "init_head.bin", dtype="<f8").size == nxy * nzd
    reg = np.fromfile(tmp_path / "region.bin", dtype="<i4").reshape(nzd, nxy)
    assert (reg[0] == -1).all() and (reg[1] == 0).all() and (reg[2:] == 1).all()
    sea = np.fromfile(tmp_path / "sea_level.bin", dtype="<f4").reshape(nzd, nxy)
    assert np.all(sea[1] == np.float32(0.55)) and np.all(sea[[0, 2, 3, 4, 5, 6]] == SNOVAL)
    grid = open(tmp_path / "grid.txt").read().split("\n")
    assert [float(v) for v in grid[3].split()] == [0.7, -0.1]        # corner at the top, downward width
    h = make_config("hetero", shape=(8, 6, 4))
    write_deck(h, str(tmp_path / "h"))
    recs = np.fromfile(tmp_path / "h" / "rain.bin", dtype="<f4").reshape(2, 49)
    assert recs[0, 0] == 6.0 and np.all(recs[0, 1:] == 20.0) and np.all(recs[1, 1:] == 0.0)
    ts = read_namelists(open(tmp_path / "h" / "timeseries.txt").read())
    assert ts["tinp_type"]["rech_type"] == 4 and ts["tinp_unit"]["rech_unit"] == "HOU"
    assert ts["tinp_type"]["rive_type"] == -1 and ts["tinp_type"]["lake_type"] == -1
    main = read_namelists(open(tmp_path / "h" / "msg123.main").read())
    assert main["set_calc_time"]["edate"] == [2000, 1, 5, 0, 0, 0]       # 96 x 3600 s after the start
    assert main["set_solution"]["criteria"] == pytest.approx(1e-8 * 0.375)   # relative 1e-8 x max|h0| (m)


def test_refusals(tmp_path):
    with pytest.raises(ValueError, match="free drainage"):
        write_deck(make_config("box", shape=(4, 4, 5)), str(tmp_path))
    p = make_config("box1r", shape=(4, 4, 5), lin_tol=1e-10)
    with pytest.raises(ValueError, match="linear tolerance"):
        write_deck(p, str(tmp_path))
    with pytest.raises(ValueError, match="nx = ny"):
        write_deck(make_config("box1r", shape=(5, 4, 5)), str(tmp_path))


@pytest.mark.parametrize("name,kw", [("hetero", dict(shape=(10, 8, 6), nsteps=3)),
                                     ("box1r", dict(shape=(4, 4, 6), nsteps=3))])
def test_oracle_runs_the_deck(tmp_path, name, kw):
    """The oracle advances the generated problem and the one read from its deck with the
    same settings (the deck's: the reference's AMG or DILU, absolute criteria, its end
    time): the same accepted steps and Newton counts, heads within 1e-6 -- the two differ
    only by the rounding of the initial heads (the reference scales them in real(DP), the
    generator in real(SP)) and, for 0.1-m cells, of the elevations."""
    p = make_config(name, **kw)
    write_deck(p, str(tmp_path))
    q = read_deck(str(tmp_path))
    S = {k: q.params[k] for k in ("precon_type", "ref_quirks", "criteria", "criteria_rel", "lin_tol", "sim_type",
                                  "ini_step", "max_step", "inc_fact", "maxout_iter", "maxinn_iter", "end_time")}
    o1, o2 = Oracle(p, **S), Oracle(q, **S)
    o1.init_state(); o2.init_state()
    r1, s1 = o1.advance(nsteps=3)
    r2, s2 = o2.advance(nsteps=3)
    assert r1 == r2 == 0 and s1["accepted"] == s2["accepted"] == 3
    assert s1["newton_total"] == s2["newton_total"]
    err = rel(o1.get_state()["head_new"], o2.get_state()["head_new"])
    print(name, s1, err)
    assert err <= 1e-6
    o1.close(); o2.close()
