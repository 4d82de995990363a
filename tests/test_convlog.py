"""Convergence log in the reference's format (Nonlinear_solution.f90:59-66,77,240-290).

CPU: the Fortran edit descriptors (ESw.d, Iw, Aw), the header and iteration line layout,
the cell label of get_cnum, and a write -> read round trip.  GPU: the library records one
entry per Newton iteration, ending with the solve's status, and the last entry agrees
with the solve's statistics and the state."""
import pytest

from msg123_b200 import convlog
from msg123_b200.config import make_config


@pytest.mark.parametrize("x,w,d,expect", [
    (0.0, 12, 3, "   0.000E+00"),
    (-1.5e-5, 12, 3, "  -1.500E-05"),
    (123456.0, 12, 5, " 1.23456E+05"),
    (9.9996e-3, 12, 3, "   1.000E-02"),
    (1.2345e150, 12, 3, "   1.234+150"),
    (-2.5e-120, 12, 3, "  -2.500-120"),
    (float("nan"), 12, 3, "         NaN"),
    (float("-inf"), 12, 3, "   -Infinity"),
    (1.0e5, 6, 3, "******"),
])
def test_es_edit_descriptor(x, w, d, expect):
    assert convlog.es(x, w, d) == expect


def test_integer_and_character_descriptors():
    assert convlog.iw(12, 6) == "    12" and convlog.iw(1234567, 6) == "******"
    assert convlog.aw("(3,2,1)", 18) == " " * 11 + "(3,2,1)"
    assert convlog.aw("x" * 20, 18) == "x" * 18


def test_cell_label_follows_get_calc_grid():
    nx, ny = 5, 4
    assert convlog.cell_label(1, nx, ny) == "(1,1,1)"
    assert convlog.cell_label(5, nx, ny) == "(5,1,1)"
    assert convlog.cell_label(6, nx, ny) == "(1,2,1)"
    assert convlog.cell_label(nx * ny + 7, nx, ny) == "(2,2,2)"


def _recs():
    base = dict(time=1800.0, delt=1800.0, in_iter=3, back_iter=0, dmat=-1.25e-3, rhs=4.5e-9, head=-9.87)
    return [dict(base, out_iter=1, cell=47, maxvar=0.125, status=-1),
            dict(base, out_iter=2, cell=47, maxvar=-3.5e-4, status=-1),
            dict(base, out_iter=3, cell=48, maxvar=2.0e-9, status=0),
            dict(base, time=3600.0, out_iter=1, cell=12, maxvar=0.5, status=convlog.MSG_LINESEARCH_FAIL)]


def test_layout_and_round_trip(tmp_path):
    nx, ny = 5, 4
    out = convlog.lines(_recs(), nx, ny)
    assert out[:2] == ["", ""]
    assert out[2] == " CURRENT TIME :  1.80000E+03 (SEC)" + " " * 20 + "TIME STEP :  1.80000E+03 (SEC)"
    assert out[3] == " " + "-" * 84 and out[4] == " " + convlog.TITLE1 and out[6] == " " + "-" * 84
    first = out[7]
    assert len(first) == 85
    assert first == ("      1     3     0   1.250E-01" + "(2,2,3)".rjust(18)
                     + "  -1.250E-03   4.500E-09  -9.870E+00")
    assert out[-1] == convlog.MESSAGES[convlog.MSG_LINESEARCH_FAIL]
    p = tmp_path / "conv.txt"
    convlog.write(p, _recs(), nx, ny)
    back = convlog.read(p)
    assert [r["out_iter"] for r in back] == [1, 2, 3, 1]
    assert [r["cell"] for r in back] == ["(2,2,3)", "(2,2,3)", "(3,2,3)", "(2,3,1)"]
    assert back[1]["maxvar"] == pytest.approx(-3.5e-4) and back[3]["time"] == pytest.approx(3600.0)
    assert back[-1]["message"] == convlog.MESSAGES[convlog.MSG_LINESEARCH_FAIL].strip()
    assert back[2]["message"] is None


@pytest.mark.gpu
def test_gpu_records_every_newton_iteration(tmp_path):
    from msg123_b200.solver import GpuSolver
    p = make_config("box", shape=(10, 9, 12), nsteps=3)
    g = GpuSolver(p)
    g.set_convlog(True)
    g.init_state()
    rc, st = g.calc_numsol()
    recs = g.convlog()
    assert rc == 0 and len(recs) == st["out_iter"]
    assert [r["out_iter"] for r in recs] == list(range(1, st["out_iter"] + 1))
    assert all(r["status"] == -1 for r in recs[:-1]) and recs[-1]["status"] == 0
    last = recs[-1]
    assert last["cell"] == st["maxnun"] and last["maxvar"] == st["maxvar"]
    ls = p.params["len_scal"]
    assert last["head"] == g.get_state()["head_new"][last["cell"] - 1] * ls
    # the time loop records every iteration of every attempt
    rc, rs = g.advance(nsteps=2)
    recs = g.convlog()
    assert rc == 0 and len(recs) == rs["newton_total"]
    assert sum(r["status"] == 0 for r in recs) == rs["accepted"]
    convlog.write(tmp_path / "conv.txt", recs, p.nx, p.ny)
    assert len(convlog.read(tmp_path / "conv.txt")) == len(recs)
    g.set_convlog(False)
    g.advance(nsteps=1)
    assert g.convlog() == []
