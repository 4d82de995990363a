"""Solver settings read from the reference's main input deck (msg123.main).

The reference reads its settings as Fortran namelist groups from msg123.main, in this order
(Read_input.f90:23-61): set_simulation, set_calc_time, set_calc_reg, set_solution (with
set_amg right after it when precon_type = 1), set_grid, then the input and output groups.
`read_namelists` parses namelist text into {group: {name: value}}; `solver_params` turns
the simulation, time and solution groups into the library's msg_params_t knobs the way
the reference turns them into its own variables, and `grid_box` reads a grid file of type 7
(corner and width per axis) into the box the library solves on.  Fields, boundary
conditions and output settings are not read here.

What follows the reference:
* set_simulation (Read_input.f90:146-180): sim_type -1 steady, 0 long-term, 1 transient;
  the library runs 0 (dt times incr_multi) and 1 (Newton-count heuristic); -1 is refused.
* set_calc_time (:182-225): calc_unit SEC/MIN/HOU/DAY/YEA sets the factor cal_fact
  (conv_unit, Utility_module.f90:322-376); sim_type 0 takes end_time * cal_fact, sim_type
  1 the seconds between sdate and edate.
* set_solution (:333-375): init_step and max_step times cal_fact (real(SP) products),
  incr_multi, maxout_iter, criteria (absolute, metres), maxinn_iter, precon_type 0 (DILU)
  or 1 (AMG; the library's reference-AMG mode, ref_quirks = 1, reproduces what the
  reference's AMG returns); set_amg (:377-395): amg_nlevel, jac_omega, amg_theta.
* set_grid (:397-426) and a type-7 grid file (:545-583): gridx/y/z cells; the file's first
  line is a header, then "corner width" for x, y and z.
"""
import datetime
import re

import numpy as np

from .config import len_scale

F32 = np.float32
_DAYSEC = 86400.0


def _strip_comment(line):
    out, q = [], None
    for ch in line:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        elif ch == "!":
            break
        else:
            out.append(ch)
    return "".join(out)


def _tokens(body):
    """Split a namelist group body into name/value tokens: strings, '=', ',' and bare words."""
    return re.findall(r"'(?:[^']|'')*'|\"(?:[^\"]|\"\")*\"|=|,|[^\s,=]+", body)


def _value(tok):
    if tok[0] in "'\"":
        return tok[1:-1].replace(tok[0] * 2, tok[0])
    t = tok.lower()
    if t in (".true.", "t", ".t."):
        return True
    if t in (".false.", "f", ".f."):
        return False
    try:
        return int(t)
    except ValueError:
        return float(t.replace("d", "e"))


def _groups(text):
    """(name, body) of each &name ... / group; a '/' or '&end' inside quotes does not close it."""
    i, n = 0, len(text)
    while True:
        m = re.compile(r"&(\w+)", re.I).search(text, i)
        if not m:
            return
        j, q = m.end(), None
        while j < n:
            ch = text[j]
            if q:
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
            elif ch == "/" or text[j:j + 4].lower() == "&end":
                break
            j += 1
        yield m.group(1).lower(), text[m.end():j]
        i = j + 1


def read_namelists(text):
    """{group: {name: value or list of values}} from Fortran namelist text (groups opened by
    &name and closed by / or &end; names case-insensitive; r*v repeat counts; ! comments)."""
    text = "\n".join(_strip_comment(l) for l in text.splitlines())
    groups = {}
    for name, body in _groups(text):
        toks = [t for t in _tokens(body) if t != ","]
        vals, key, cur = {}, None, []
        i = 0
        while i < len(toks):
            if i + 1 < len(toks) and toks[i + 1] == "=":
                if key is not None:
                    vals[key] = cur[0] if len(cur) == 1 else cur
                key, cur = toks[i].lower(), []
                i += 2
                continue
            tok = toks[i]
            rep = re.fullmatch(r"(\d+)\*(.+)", tok)
            cur += [_value(rep.group(2))] * int(rep.group(1)) if rep else [_value(tok)]
            i += 1
        if key is not None:
            vals[key] = cur[0] if len(cur) == 1 else cur
        groups[name] = vals
    return groups


def cal_fact(unit, sdate=(0, 0, 0, 0, 0, 0)):
    """conv_unit (Utility_module.f90:322-376): seconds per calculation-time unit, real(SP)."""
    u = unit.strip().upper()
    if u == "SEC":
        return float(F32(1.0))
    if u == "MIN":
        return float(F32(60.0))
    if u == "HOU":
        return float(F32(3600.0))
    if u == "DAY":
        return float(F32(_DAYSEC))
    if u == "YEA":
        year = sdate[0] if sdate[1] <= 2 else sdate[0] + 1
        leap = year != 0 and (year % 400 == 0 or (year % 100 != 0 and year % 4 == 0))
        return float(F32(_DAYSEC * (366 if leap else 365)))
    raise ValueError(f"unknown calculation time unit {unit!r}")


def solver_params(groups):
    """msg_params_t overrides (a dict for config.default_params / GpuSolver) from the
    set_simulation, set_calc_time, set_solution and set_amg groups."""
    sim = groups.get("set_simulation", {})
    sim_type = int(sim.get("sim_type", -2))
    if sim_type == -1:
        raise ValueError("steady-state runs (sim_type = -1) are not supported by the library")
    if sim_type not in (0, 1):
        raise ValueError(f"set_simulation: sim_type {sim_type} is not a simulation type")
    tm = groups.get("set_calc_time", {})
    unit = str(tm.get("calc_unit", ""))
    if not unit.strip():
        raise ValueError("set_calc_time: calc_unit is missing")
    sdate = list(tm.get("sdate", [0] * 6)) if isinstance(tm.get("sdate"), list) else [0] * 6
    fact = cal_fact(unit, sdate)
    if sim_type == 0:
        end_time = float(F32(F32(tm.get("end_time", 0.0)) * F32(fact)))
    else:
        edate = tm["edate"]
        span = datetime.datetime(*map(int, edate)) - datetime.datetime(*map(int, sdate))
        end_time = float(F32(span.total_seconds()))
    sol = groups.get("set_solution", {})
    for k in ("maxout_iter", "maxinn_iter"):
        if int(sol.get(k, 0)) <= 0:
            raise ValueError(f"set_solution: {k} must be positive")
    precon = int(sol.get("precon_type", 0))
    if precon not in (0, 1):
        raise ValueError("set_solution: precon_type must be 0 or 1")
    p = dict(sim_type=sim_type,
             ini_step=float(F32(F32(sol.get("init_step", 0.0)) * F32(fact))),
             max_step=float(F32(F32(sol.get("max_step", 0.0)) * F32(fact))),
             inc_fact=float(F32(sol.get("incr_multi", 0.0))),
             end_time=end_time,
             maxout_iter=int(sol["maxout_iter"]), maxinn_iter=int(sol["maxinn_iter"]),
             criteria=float(sol.get("criteria", 1.0e-3)), criteria_rel=0, lin_tol=0.0,
             precon_type=precon, ref_quirks=1)
    if precon == 1:
        amg = groups.get("set_amg", {})
        p.update(amg_nlevel=int(amg.get("amg_nlevel", 0)) or 10,
                 jac_omega=float(F32(amg.get("jac_omega", 0.67))),
                 amg_theta=float(F32(amg.get("amg_theta", 0.05))))
    return p


def grid_box(groups, grid_text):
    """(nx, ny, nz, widths (dx, dy, dz) in metres, len_scal) from set_grid and the text of a
    type-7 grid file (first line a header, then "corner width" for x, y and z)."""
    g = groups["set_grid"]
    if int(g.get("grid_type", -1)) != 7:
        raise ValueError("only grid_type 7 (corner and width per axis) is read here")
    nx, ny, nz = int(g["gridx"]), int(g["gridy"]), int(g["gridz"])
    lines = [l.split() for l in grid_text.splitlines() if l.strip()]
    (xc, xw), (yc, yw), (zc, zw) = [(F32(float(a)), F32(float(b))) for a, b, *_ in lines[1:4]]
    # glob_z(:,:,k) = zcorner + zwidth*(k-1), both products and the sum in real(SP)
    zs = [float(zc + zw * F32(k)) for k in range(nz + 1)]
    return nx, ny, nz, (abs(float(xw)), abs(float(yw)), abs(float(zw))), float(len_scale(max(abs(z) for z in zs)))
