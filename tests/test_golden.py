"""Committed fixtures (tests/golden, made by tests/golden/make_golden.py).

* The oracle's van Genuchten / Mualem values against the closed forms evaluated in extended
  precision, independent of any implementation (Calc_parameter.f90:15-77).  S agrees to
  1e-14 (measured 2e-16); kr to 1e-10 (measured 3e-12), because the reference's form
  cancels in 1 - (1 - Se^(1/m))^m as the soil dries (kr down to 2.5e-11 here).
* A regression fixture of the oracle itself (a 6x5x8 box after three steps): the heads and
  counts must not drift.
"""
import dataclasses
import json
import os

import numpy as np

from msg123_b200.config import make_config
from oracle.oracle import Oracle

HERE = os.path.join(os.path.dirname(__file__), "golden")


def test_oracle_against_closed_form_fixture():
    soils = json.load(open(os.path.join(HERE, "vg_closed_form.json")))
    for entry in soils:
        s, vals = entry["soil"], entry["values"]
        n = len(vals)
        p = make_config("box", shape=(n, 1, 1))
        assert p.params["len_scal"] == 1.0              # lengths stay in metres
        f32 = lambda v: np.full(n, v, dtype=np.float32)
        p = dataclasses.replace(p, reta=f32(s["alpha"]), retn=f32(s["n"]), resi=f32(s["thr"]), poro=f32(s["ths"]))
        psi = np.array([v["psi"] for v in vals])
        S, kr, _ = Oracle(p).srat_rperm(p.cell_top + psi)
        want_s = np.array([v["S"] for v in vals])
        want_k = np.array([v["kr"] for v in vals])
        assert np.max(np.abs(S - want_s) / want_s) < 1e-14
        assert np.max(np.abs(kr - want_k) / want_k) < 1e-10


def test_oracle_box_run_regression():
    g = np.load(os.path.join(HERE, "oracle_box_run.npz"))
    p = make_config("box", shape=(6, 5, 8), nsteps=3)
    o = Oracle(p)
    o.init_state()
    rc, st = o.advance(nsteps=3)
    assert rc == int(g["rc"]) and st["newton_total"] == int(g["newton"]) and st["krylov_total"] == int(g["krylov"])
    assert st["current_t"] == float(g["t"])
    assert np.array_equal(o.get_state()["head_new"], g["head"])
