"""The reference's convergence log, written from the library's per-iteration records.

msg_gpu_set_convlog / msg_gpu_convlog (GpuSolver.set_convlog / .convlog) record one entry
per Newton iteration; this module writes them as the reference's conv file
(Nonlinear_solution.f90:59-66, header at :77, one line per iteration at :240-252, the
closing messages at :256-290) and reads such a file back, so that a run of this library
and a run of the Fortran build can be compared line by line.

Formats reproduced:
  10  (//1x,"CURRENT TIME : ",es12.5,1x,"(",a,")",20x,"TIME STEP : ",es12.5,1x,"(SEC)",
       /,1x,84("-"),/,1x, column titles (two records),/,1x,84("-"))
  11  (1X,3(i6),es12.3,a18,4(es12.3))   outer, inner, back, change, "(i,j,k)", diag, rhs, head
  12, 13, 14  the messages after a diverged, line-search-failed or capped Newton solve
"""
import math

MSG_OK, MSG_NEWTON_MAXIT, MSG_NAN, MSG_LINESEARCH_FAIL, MSG_DIVERGED = 0, 1, 2, 3, 4

TITLE1 = " OUTER INNER  BACK     MAXIMUM           MAXIMUM    DIAGONAL  RIGHT HAND     UNKNOWN"
TITLE2 = "                        CHANGE              CELL      MATRIX      VECTOR       VALUE"
MESSAGES = {
    MSG_DIVERGED: " Didn't converge due to maximum value or change",          # format 12
    MSG_LINESEARCH_FAIL: " Stop due to maximum value or change in backtracking",  # format 13
    MSG_NEWTON_MAXIT: " Stop due to maximum number of nonlinear iteration",    # format 14
}


def es(x, w, d):
    """Fortran ESw.d output of a real: one nonzero digit before the point, d after it,
    exponent E+dd (or +ddd from 100 on), right-justified in w; w asterisks if it does
    not fit."""
    if math.isnan(x):
        s = "NaN"
    elif math.isinf(x):
        s = "-Infinity" if x < 0 else "Infinity"
    else:
        mant, ex = f"{x:.{d}E}".split("E")
        e = int(ex)
        s = mant + (f"E{e:+03d}" if abs(e) <= 99 else f"{e:+04d}")
    return s.rjust(w) if len(s) <= w else "*" * w


def iw(n, w):
    """Fortran Iw output."""
    s = str(int(n))
    return s.rjust(w) if len(s) <= w else "*" * w


def aw(s, w):
    """Fortran Aw output of a character value: right-justified when shorter, the leading
    w characters when longer."""
    return s.rjust(w) if len(s) <= w else s[:w]


def cell_label(cell, nx, ny):
    """get_cnum / get_calc_grid (Nonlinear_solution.f90:737-758, Set_cell.f90:1345-1363) for a
    grid whose cells are all active: 1-based cell number -> "(i,j,k)"."""
    z = (cell - 1) // (nx * ny) + 1
    xy = cell - nx * ny * (z - 1)
    y = (xy - 1) // nx + 1
    x = xy - (y - 1) * nx
    return f"({x},{y},{z})"


def header(time, delt, unit="SEC"):
    """Format 10: the records written at the first Newton iteration of a solve."""
    return ["", "",
            " CURRENT TIME : " + es(time, 12, 5) + " (" + unit + ")" + " " * 20 + "TIME STEP : " + es(delt, 12, 5)
            + " (SEC)",
            " " + "-" * 84, " " + TITLE1, " " + TITLE2, " " + "-" * 84]


def line(rec, nx, ny):
    """Format 11: one Newton iteration."""
    return (" " + iw(rec["out_iter"], 6) + iw(rec["in_iter"], 6) + iw(rec["back_iter"], 6) + es(rec["maxvar"], 12, 3)
            + aw(cell_label(rec["cell"], nx, ny), 18) + es(rec["dmat"], 12, 3) + es(rec["rhs"], 12, 3)
            + es(rec["head"], 12, 3))


def lines(records, nx, ny, unit="SEC", seconds_per_unit=1.0):
    """The log lines of a sequence of records (GpuSolver.convlog()), in the reference's
    order: a header at each solve's first iteration, one line per iteration, and the
    closing message of a solve that ended without converging."""
    out = []
    for r in records:
        if r["out_iter"] == 1:
            out.extend(header(r["time"] / seconds_per_unit, r["delt"], unit))
        out.append(line(r, nx, ny))
        if r["status"] in MESSAGES:
            out.append(MESSAGES[r["status"]])
    return out


def write(path, records, nx, ny, unit="SEC", seconds_per_unit=1.0, mode="w"):
    with open(path, mode) as f:
        for s in lines(records, nx, ny, unit, seconds_per_unit):
            f.write(s + "\n")


def _real(s):
    """A real written by ESw.d, including the E-less form of 3-digit exponents."""
    s = s.strip()
    if "E" in s or s in ("NaN", "Infinity", "-Infinity"):
        return float(s.replace("Infinity", "inf"))
    k = max(s.rfind("+"), s.rfind("-"))
    return float(s[:k] + "E" + s[k:])


def read(path):
    """Parse a conv file written by the reference (or by `write`): a list of
    {time, delt, out_iter, in_iter, back_iter, cell, maxvar, dmat, rhs, head} with the
    cell as the "(i,j,k)" label, and the closing message (or None) of each solve."""
    recs = []
    time = delt = None
    with open(path) as f:
        for s in f:
            s = s.rstrip("\n")
            if s.startswith(" CURRENT TIME : "):
                time = _real(s[16:28])
                k = s.index("TIME STEP : ") + 12
                delt = _real(s[k:k + 12])
                continue
            if s in MESSAGES.values():
                if recs:
                    recs[-1]["message"] = s.strip()
                continue
            if len(s) >= 85 and s[1:7].strip().isdigit():
                recs.append(dict(time=time, delt=delt, out_iter=int(s[1:7]), in_iter=int(s[7:13]),
                                 back_iter=int(s[13:19]), maxvar=_real(s[19:31]), cell=s[31:49].strip(),
                                 dmat=_real(s[49:61]), rhs=_real(s[61:73]), head=_real(s[73:85]), message=None))
    return recs
