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
