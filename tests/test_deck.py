"""Solver settings from the reference's main deck (msg123.main): the namelist parser, the
mapping of set_simulation / set_calc_time / set_solution / set_amg onto the library's
knobs (Read_input.f90:146-395, conv_unit in Utility_module.f90:322-376) and a type-7 grid
(:545-583); the knobs then drive the oracle."""
import numpy as np
import pytest

from msg123_b200 import deck
from msg123_b200.config import default_params, make_config

MAIN = """
! a main deck written for this test
&set_simulation sim_type = 1, sim_name = 'hill slope' /
&set_calc_time stime_type = 0, sdate = 2021, 3, 1, 0, 0, 0,
   edate = 2021 3 3 0 0 0, calc_unit = "HOU" /
&set_calc_reg calc_type = 7, calcreg_neib = 1 /
&SET_SOLUTION
  init_step = 0.5, incr_multi = 1.0, max_step = 2.0   ! hours
  maxout_iter = 20, criteria = 1.0d-4, maxinn_iter = 50, precon_type = 1
/
&set_amg amg_nlevel = 6, maxvcy_iter = 1, max_sweep = 2, jac_omega = 0.6, amg_theta = 0.08 /
&set_grid gridx = 16, gridy = 12, gridz = 8, grid_type = 7, grid_file = 'grid.txt' /
&misc flags = 3*.true., .false., name = 'it''s' /
"""


def test_namelist_parser():
    g = deck.read_namelists(MAIN)
    assert g["set_simulation"] == {"sim_type": 1, "sim_name": "hill slope"}
    assert g["set_calc_time"]["sdate"] == [2021, 3, 1, 0, 0, 0] and g["set_calc_time"]["edate"][2] == 3
    assert g["set_calc_time"]["calc_unit"] == "HOU"
    assert g["set_solution"]["criteria"] == 1.0e-4 and g["set_solution"]["maxinn_iter"] == 50
    assert g["misc"] == {"flags": [True, True, True, False], "name": "it's"}
    # a '/' or '!' inside quotes neither closes the group nor starts a comment; &end closes too
    h = deck.read_namelists("&set_grid grid_file = 'in/grid!1.txt', gridx = 2 /\n"
                            "&set_calc_time sdate = 6*0, end_time = 3.6d3 &end\n&set_simulation sim_type=0/")
    assert h["set_grid"] == {"grid_file": "in/grid!1.txt", "gridx": 2}
    assert h["set_calc_time"] == {"sdate": [0] * 6, "end_time": 3600.0} and h["set_simulation"] == {"sim_type": 0}


def test_solver_params_from_a_transient_deck():
    p = deck.solver_params(deck.read_namelists(MAIN))
    assert p["sim_type"] == 1 and p["ini_step"] == 1800.0 and p["max_step"] == 7200.0
    assert p["end_time"] == 2 * 86400.0 and p["inc_fact"] == 1.0
    assert (p["maxout_iter"], p["maxinn_iter"], p["criteria"], p["criteria_rel"]) == (20, 50, 1.0e-4, 0)
    assert p["precon_type"] == 1 and p["ref_quirks"] == 1 and p["amg_nlevel"] == 6
    assert p["jac_omega"] == float(np.float32(0.6)) and p["amg_theta"] == float(np.float32(0.08))
    assert set(p) <= set(default_params())              # every knob is a msg_params_t field


def test_long_term_deck_and_errors():
    base = "&set_simulation sim_type = 0 /\n&set_calc_time end_time = 10, calc_unit = 'DAY' /\n"
    sol = "&set_solution init_step = 0.25, incr_multi = 1.5, maxout_iter = 10, maxinn_iter = 10 /\n"
    p = deck.solver_params(deck.read_namelists(base + sol))
    assert p["end_time"] == 864000.0 and p["ini_step"] == 21600.0 and p["inc_fact"] == 1.5
    assert p["precon_type"] == 0 and p["criteria"] == 1.0e-3       # the reference's default
    assert deck.cal_fact("YEA", (2024, 1, 1, 0, 0, 0)) == 366 * 86400.0
    assert deck.cal_fact("YEA", (2023, 6, 1, 0, 0, 0)) == 366 * 86400.0   # after February: next year
    with pytest.raises(ValueError, match="steady"):
        deck.solver_params(deck.read_namelists(base.replace("sim_type = 0", "sim_type = -1") + sol))
    with pytest.raises(ValueError, match="calc_unit"):
        deck.solver_params(deck.read_namelists("&set_simulation sim_type = 0 /\n&set_calc_time /\n" + sol))
    with pytest.raises(ValueError, match="precon_type"):
        deck.solver_params(deck.read_namelists(base + sol.replace("maxinn_iter = 10", "maxinn_iter = 10, "
                                                                  "precon_type = 2")))


def test_grid_box_and_a_run_with_the_deck_knobs():
    g = deck.read_namelists(MAIN)
    nx, ny, nz, widths, ls = deck.grid_box(g, "corner width\n 0.0 1.0\n 0.0 1.0\n -2.0 0.25\n")
    assert (nx, ny, nz) == (16, 12, 8) and widths == (1.0, 1.0, 0.25) and ls == 10.0   # max|z| = 2 m
    nx, ny, nz, widths, ls = deck.grid_box(g, "h\n0 1\n0 1\n-16 2\n")
    assert ls == 100.0                                   # max|z| = 16 m -> 10^2
    from oracle.oracle import Oracle
    knobs = deck.solver_params(g)
    knobs.update(precon_type=0)                          # DILU keeps this check quick
    p = make_config("hetero", shape=(nx, ny, nz), seed=5, **knobs)
    o = Oracle(p)
    o.init_state()
    rc, st = o.advance(nsteps=2)
    assert rc == 0 and st["accepted"] == 2 and st["current_t"] > 0
