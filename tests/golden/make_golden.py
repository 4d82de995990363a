"""Writes the fixtures of tests/golden (run from the repository root:
`python tests/golden/make_golden.py`).

* vg_closed_form.json -- van Genuchten saturation and Mualem kr at chosen pressure heads
  for two soils, evaluated from the closed forms (Calc_parameter.f90:15-77) in numpy's
  extended precision (float128 on x86-64): independent of the library and the oracle.
* oracle_box_run.npz -- heads and step statistics of the oracle on a 6x5x8 box after three
  steps: a regression fixture of the C restatement (not of the reference, which ships no
  vectors), so that any drift of the oracle shows.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

SOILS = [dict(alpha=3.35, n=2.0, thr=0.102, ths=0.368), dict(alpha=1.2, n=1.45, thr=0.05, ths=0.41)]
PSI = [-1e-3, -0.05, -0.3, -1.0, -3.0, -10.0, -50.0]


def vg_closed_form():
    L = np.longdouble
    out = []
    for s in SOILS:
        a, n = L(np.float32(s["alpha"])), L(np.float32(s["n"]))
        thr, ths = L(np.float32(s["thr"])), L(np.float32(s["ths"]))
        # theta_s - theta_r is a real(SP) difference in the reference, so it is taken in float32
        dth = L(np.float32(s["ths"]) - np.float32(s["thr"]))
        m = L(1) - L(1) / n
        rows = []
        for psi in PSI:
            se = (L(1) + abs(a * L(psi)) ** n) ** (-m)
            kr = np.sqrt(se) * (L(1) - (L(1) - se ** (L(1) / m)) ** m) ** 2
            rows.append(dict(psi=psi, S=float((thr + dth * se) / ths), kr=float(kr)))
        out.append(dict(soil=s, values=rows))
    return out


def oracle_box_run():
    from msg123_b200.config import make_config
    from oracle.oracle import Oracle
    p = make_config("box", shape=(6, 5, 8), nsteps=3)
    o = Oracle(p)
    o.init_state()
    rc, st = o.advance(nsteps=3)
    return dict(head=o.get_state()["head_new"], rc=rc, newton=st["newton_total"], krylov=st["krylov_total"],
                t=st["current_t"])


if __name__ == "__main__":
    with open(os.path.join(HERE, "vg_closed_form.json"), "w") as f:
        json.dump(vg_closed_form(), f, indent=1)
    np.savez(os.path.join(HERE, "oracle_box_run.npz"), **oracle_box_run())
