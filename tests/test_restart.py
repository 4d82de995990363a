"""Checkpoint / resume through the reference's restart file (gfortran sequential
unformatted: [int32 8][real(DP) time][int32 8] [int32 8n][n x real(DP) head*len_scal][int32 8n],
Nonlinear_solution.f90:792-816; read back with head = value * len_scal_inv, the reciprocal
taken in single precision, Read_input.f90:1108, Assign_calculation.f90:416-434)."""
import struct

import numpy as np
import pytest

from msg123_b200.config import make_config
from msg123_b200.solver import read_restart


def _fortran_file(path, t, vals):
    with open(path, "wb") as f:
        f.write(struct.pack("<i", 8) + struct.pack("<d", t) + struct.pack("<i", 8))
        b = np.ascontiguousarray(vals, dtype="<f8").tobytes()
        f.write(struct.pack("<i", len(b)) + b + struct.pack("<i", len(b)))


def test_read_restart_written_like_gfortran(tmp_path):
    rng = np.random.default_rng(0)
    vals = rng.uniform(-20.0, 5.0, 1000)
    ls = 10.0
    p = tmp_path / "rest.bin"
    _fortran_file(p, 3600.0, vals)
    h, t = read_restart(p, 1000, ls)
    assert t == 3600.0
    # value * len_scal_inv with the reciprocal taken in single precision, as assign_initv does
    assert np.array_equal(h, vals * np.float64(np.float32(1.0) / np.float32(ls)))
    with pytest.raises(RuntimeError):
        read_restart(p, 999, ls)          # record length does not match the grid
    (tmp_path / "short.bin").write_bytes(p.read_bytes()[:100])
    with pytest.raises(RuntimeError):
        read_restart(tmp_path / "short.bin", 1000, ls)


@pytest.mark.gpu
def test_write_restart_and_resume(tmp_path):
    from msg123_b200.solver import GpuSolver
    p = make_config("box", shape=(8, 6, 10), nsteps=4)
    g = GpuSolver(p)
    g.init_state()
    g.advance(nsteps=2)
    path = tmp_path / "rest.bin"
    g.write_restart(path)
    raw = path.read_bytes()
    n = p.ncalc
    assert len(raw) == 8 + 8 + 8 + 8 * n
    assert struct.unpack_from("<i", raw, 0)[0] == 8 and struct.unpack_from("<i", raw, 12)[0] == 8
    assert struct.unpack_from("<i", raw, 16)[0] == 8 * n and struct.unpack_from("<i", raw, 20 + 8 * n)[0] == 8 * n
    h_dev = g.get_state()["head_new"]
    ls = p.params["len_scal"]
    assert np.array_equal(np.frombuffer(raw, "<f8", n, 20), h_dev * ls)
    h, t = read_restart(path, n, ls)
    assert t == 3600.0
    assert np.array_equal(h, (h_dev * ls) * np.float64(np.float32(1.0) / np.float32(ls)))
    # resume: a new context started from the restart heads continues the run
    g2 = GpuSolver(p)
    g2.init_state(head=h)
    rc, st = g2.advance(nsteps=2)
    assert rc == 0 and st["accepted"] == 2
