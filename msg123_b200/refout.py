"""Files in the reference's binary formats: output series written from the library's state,
and the plain real(SP) fields its input decks use.

The reference writes its head, saturation and water-table files as unformatted stream
files (open_new_wbin, Utility_module.f90:156-184): for each output time one record of
  real(SP) time                                  (write_header_bin, Write_module.f90:207-225)
  real(SP) field(nx, ny[, nz]), x fastest        (write_3dbin :146-185, write_2dbin :61-99)
where each active cell holds real(value * unit, SP) -- the product taken in double, the
unit being len_scal for heads and the water table and 1 for saturation -- and every other
entry SNOVAL = -9999.  Cell c (1-based, local order: x fastest, then y, layers from the top)
lands at (x, y, z) = get_calc_grid(c) (Set_cell.f90:1345-1363), so on a grid whose cells are
all active the field is the state vector itself.  The series are written by
write_out_headf (Write_output.f90:321-366, unit len_scal), write_out_sratf (:368-413, unit
1) and write_out_wtabf (:434-496, unit len_scal, field from calc_wtable).

`append` adds one record, `read` returns the records of a file written here or by the
Fortran build, and `write_state` writes the three series for a solver's current state.

Input fields of type 6 (3D) and 4 (2D) are the same stream layout without the time
header: read_3d_r4bin / read_2d_r4bin (Read_module.f90:266-299,446-479) read
real(SP) field(nx, ny[, nz]) x fastest, and set_3dr4_calc (Set_condition.f90:1092-1160) hands value
(x, y, z) to the cell of that grid position -- on a full grid, the local cell order.
`write_field` / `read_field` write and read them.
"""
import numpy as np

SNOVAL = np.float32(-9999.0)


def field(values, unit, shape):
    """The real(SP) array write_3dbin / write_2dbin emits for `values` (local cell order,
    every cell active): float32(value * unit) with the product in double, x fastest."""
    v = np.asarray(values, dtype=np.float64).reshape(-1)
    n = int(np.prod(shape))
    if v.size != n:
        raise ValueError(f"field: {v.size} values for a {shape} grid")
    return (v * np.float64(np.float32(unit))).astype(np.float32)


def append(path, time, values, unit, shape):
    """Append one record (time, field) to a series file; shape = (nx, ny) or (nx, ny, nz)."""
    with open(path, "ab") as f:
        f.write(np.float32(time).tobytes())
        f.write(field(values, unit, shape).astype("<f4").tobytes())


def read(path, shape):
    """All records of a series file: a list of (time, float32 array of `shape` reversed,
    i.e. [nz, ny, nx] or [ny, nx]); SNOVAL marks inactive cells."""
    n = int(np.prod(shape))
    raw = np.fromfile(path, dtype="<f4")
    if raw.size % (n + 1):
        raise ValueError(f"read: {path} is not a series of {shape} records")
    recs = raw.reshape(-1, n + 1)
    return [(float(r[0]), r[1:].reshape(tuple(reversed(shape)))) for r in recs]


def write_field(path, values, shape):
    """An input field of type 6 (shape (nx, ny, nz)) or 4 (shape (nx, ny)): the values as
    real(SP), local cell order = x fastest, no header."""
    v = np.asarray(values, dtype=np.float32).reshape(-1)
    if v.size != int(np.prod(shape)):
        raise ValueError(f"write_field: {v.size} values for a {shape} grid")
    v.astype("<f4").tofile(path)


def read_field(path, shape):
    """An input field written by `write_field` (or for the Fortran build), as a float32
    array of `shape` reversed ([nz, ny, nx] or [ny, nx])."""
    raw = np.fromfile(path, dtype="<f4")
    if raw.size != int(np.prod(shape)):
        raise ValueError(f"read_field: {path} holds {raw.size} values, not a {shape} grid")
    return raw.reshape(tuple(reversed(shape)))


def ew(x, w=13, d=6):
    """Fortran Ew.d output of a real (OUTFORM = "(E13.6)", Constval_module.f90:30): 0.ddd…
    with d digits, exponent E+xx (or +xxx from 100 on), right-justified in w; w asterisks
    when it does not fit."""
    x = float(x)
    if x != x:
        s = "NaN"
    elif x in (float("inf"), float("-inf")):
        s = "-Infinity" if x < 0 else "Infinity"
    elif x == 0.0:
        s = "0." + "0" * d + "E+00"
    else:
        mant, ex = f"{abs(x):.{d - 1}E}".split("E")
        e = int(ex) + 1
        s = ("-" if x < 0 else "") + "0." + mant.replace(".", "") + (f"E{e:+03d}" if abs(e) <= 99 else f"{e:+04d}")
    return s.rjust(w) if len(s) <= w else "*" * w


class MassBalance:
    """The reference's whole-area mass-balance file (mass type 7, one region "whole area"):
    write_mass_header (Write_output.f90:284-318) writes
        <calc unit>,whole area
        ,FLOW,STORAGE,RECHARGE,WELL,SURFACE,RIVER,LAKE,SEA,ALL
    calc_cell_mas (Calc_output.f90:54-91) adds every time step's volumes, and at each output
    time write_out_massf (Write_output.f90:498-538) scales them by len_scal**3 (a
    single-precision product), calc_out_mass (Calc_output.f90:93-166) sums them and ALL,
    and one line "time,FLOW,...,ALL" is written in E13.6, after which the sums restart.

    Feed it msg_gpu_calc_mass's nine volumes after every accepted step (`add_step`) and
    call `write(time_out)` at output times.  The ninth volume, free drainage through the
    bottom (an extension without a reference column), is added into ALL only."""

    COLUMNS = "FLOW,STORAGE,RECHARGE,WELL,SURFACE,RIVER,LAKE,SEA,ALL"

    def __init__(self, path, cal_unit, len_scal):
        self.path = path
        lf = np.float32(len_scal)
        self.cubic = float(lf * lf * lf)
        self.acc = np.zeros(9)
        with open(path, "w") as f:
            f.write(f"{cal_unit.strip()},whole area\n,{self.COLUMNS}\n")

    def add_step(self, volumes):
        """One step's calc_mass volumes: storage, flow, recharge, well, surface, river,
        lake, sea, drainage."""
        v = np.asarray(volumes, dtype=np.float64)
        if v.size != 9:
            raise ValueError("add_step: nine volumes expected")
        self.acc += v

    def write(self, time_out):
        sto, con, rec, wel, sur, riv, lak, sea, drn = self.acc * self.cubic
        tot = sto + con + sea + wel + rec + sur + riv + lak + drn
        vals = [con, sto, rec, wel, sur, riv, lak, sea, tot]
        line = ew(np.float32(time_out)) + "".join("," + ew(v) for v in vals)
        with open(self.path, "a") as f:
            f.write(line + "\n")
        self.acc[:] = 0.0
        return line


def read_mass(path):
    """Rows of a mass-balance file (this writer's or the Fortran build's) as dicts of time
    and the nine columns."""
    with open(path) as f:
        lines = f.read().splitlines()
    cols = lines[1].split(",")[1:10]
    rows = []
    for s in lines[2:]:
        v = [float(t.replace("E", "e")) if "E" in t else _fortran_real(t) for t in s.split(",")]
        rows.append(dict(time=v[0], **{c: x for c, x in zip(cols, v[1:10])}))
    return rows


def _fortran_real(t):
    """A real written without its E (exponent of three digits)."""
    t = t.strip()
    k = max(t.rfind("+"), t.rfind("-"))
    return float(t[:k] + "e" + t[k:]) if k > 0 else float(t)


def write_state(prefix, solver, time, len_scal):
    """Append the current head (unit len_scal), saturation (unit 1) and water table (unit
    len_scal, computed on the device) of `solver` to prefix + '_head.bin', '_srat.bin' and
    '_wtab.bin' as one record at output time `time`."""
    p = solver.prob
    st = solver.get_state()
    append(prefix + "_head.bin", time, st["head_new"], len_scal, (p.nx, p.ny, p.nz))
    append(prefix + "_srat.bin", time, st["srat_new"], 1.0, (p.nx, p.ny, p.nz))
    append(prefix + "_wtab.bin", time, solver.water_table(), len_scal, (p.nx, p.ny))
    return st
