"""Solver settings read from the reference's main input deck (msg123.main).

The reference reads its settings as Fortran namelist groups from msg123.main, in this order
(Read_input.f90:23-61): set_simulation, set_calc_time, set_calc_reg, set_solution (with
set_amg right after it when precon_type = 1), set_grid, then the input and output groups.
`read_namelists` parses namelist text into {group: {name: value}}; `solver_params` turns
the simulation, time and solution groups into the library's msg_params_t knobs the way
the reference turns them into its own variables, and `grid_box` reads a grid file of type 7
(corner and width per axis) into the box the library solves on.  `write_deck` writes a
generated problem as a whole deck (msg123.main, grid, field, initial-head, region and
time-series files) that the reference's own build reads, and `read_deck` reads such a deck
back into a problem, fields, boundaries and all, scaled as the reference scales them.

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


# ---------------------------------------------------------------------------------------
# Writing a deck: msg123.main and the files it names, for a generated problem
# ---------------------------------------------------------------------------------------
SNOVAL = -9999.0          # the reference's "no value" (Constval_module.f90:21,25)
_SDATE = (2000, 1, 1, 0, 0, 0)


def _fmt(v):
    if isinstance(v, str):
        return "'" + v.replace("'", "''") + "'"
    if isinstance(v, bool):
        return ".true." if v else ".false."
    if isinstance(v, (list, tuple)):
        return ", ".join(_fmt(x) for x in v)
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return repr(float(v)).replace("e", "E")


def namelist(name, **vals):
    """One namelist group in the text form gfortran reads (&name, one name = value per line, /)."""
    body = "".join(f"  {k} = {_fmt(v)}\n" for k, v in vals.items())
    return f"&{name}\n{body}/\n"


def _r4(path, arr):
    np.asarray(arr, dtype="<f4").tofile(path)


def write_deck(p, directory, end_time=None, sim_name="synthetic", outputs=("srat", "wtab", "mass"),
               out_hours=1):
    """Write msg123.main and the files it names into `directory` for a generated problem
    (config.make_config), so that the reference's own build reads the same problem:

    * set_simulation / set_calc_time (Read_input.f90:148-225): sim_type as in the problem,
      time in seconds (calc_unit SEC); sim_type 1 runs from 2000-01-01 00:00:00 to the end
      date end_time seconds later;
    * set_calc_reg (:227-267): the whole grid (calc_type 0), or for a ponded top a 3D int32
      region file (calc_type 6: -1 an inactive layer, 0 the sea layer, 1 the soil below --
      the reference stops unless some cell is -1, Set_cell.f90:505-507);
    * set_solution / set_amg (:337-395): steps in seconds, maxout_iter, maxinn_iter,
      precon_type, criteria in metres (a relative criterion becomes criteria * max|h0|),
      amg_nlevel, jac_omega, amg_theta;
    * set_grid and a type-7 grid file (:397-583): corner and width per axis, z from the top
      down (negative width);
    * set_retn_parm (:618-663): compile files (inretn_type / inretn_path, inparm_type /
      inparm_path, Open_file.f90:34-300) naming 3D float32 stream files (in_type 6) of
      alpha, n, residual content, Ks x/y/z, Ss and saturated content, x fastest, top layer
      first (Read_module.f90:459-485, flat_3d_3dr4);
    * set_init (:665-713): the initial heads as a 3D float64 stream file (init_type 6);
    * set_time_input: a time-series file (tinp_type / tinp_path / tinp_unit, :715-880)
      with the rain as 2D float32 records in mm/h (rech_type 4, unit HOU: each record is its
      float32 end time in hours followed by the field, Read_module.f90:skip_file), and the
      sea head of a ponded top as a 3D float32 field, -9999 outside the sea layer (seal_type
      6, no unit: constant);
    * set_geog off, set_wtab 7, set_mass 7 (whole area), outputs every out_hours hours.

    Refused (no counterpart in a deck): free drainage at the bottom and a fixed linear
    tolerance.  Returns the list of files written."""
    import os
    ph = p.phys
    if ph is None:
        raise ValueError("the problem carries no unscaled inputs (phys)")
    if p.free_drainage:
        raise ValueError("free drainage at the bottom has no counterpart in a reference deck")
    prm = p.params
    if prm.get("lin_tol", 0.0) != 0.0:
        raise ValueError("a fixed linear tolerance (lin_tol) has no counterpart in a reference deck")
    os.makedirs(directory, exist_ok=True)
    nx, ny, nz = p.nx, p.ny, p.nz
    extra = 2 if p.sea_top else 0                   # inactive layer + sea layer above the soil
    nzd = nz + extra
    dx, dy, dz = ph["dx"], ph["dy"], ph["dz"]
    z_grid = ph["z_top"] + extra * dz
    if float(len_scale(z_grid)) != float(prm["len_scal"]):
        raise ValueError("the deck's grid would change len_scal")
    if extra and nx != ny:
        # read_3d_calcreg places cell (i, j, k) at nx*ny*(k-1) + ny*(j-1) + i
        # (Read_module.f90:1236), the grid index only when nx = ny
        raise ValueError("a region file (ponded top) is read correctly by the reference only for nx = ny")
    files = []
    J = lambda name: os.path.join(directory, name)

    def put(name, text):
        with open(J(name), "w") as f:
            f.write(text)
        files.append(name)

    def field3d(vals, fill):
        full = np.empty(nx * ny * nzd, dtype=np.float64)
        full[: extra * nx * ny] = fill
        full[extra * nx * ny:] = vals
        return full

    # grid (type 7): header, then "corner width" for x, y (southward) and z (downward)
    put("grid.txt", "corner width\n" + f"0.0 {dx!r}\n" + f"0.0 {dy!r}\n" + f"{z_grid!r} {-dz!r}\n")
    # fields: the extra layers above the soil repeat the top soil layer's values
    top = lambda a: np.tile(np.asarray(a)[: nx * ny], extra) if extra else np.zeros(0)
    for key in ("alpha", "n", "resi", "ksx", "ksy", "ksz", "ss", "ths"):
        a = np.asarray(ph[key], dtype=np.float32)
        _r4(J(key + ".bin"), np.concatenate([top(a), a]))
        files.append(key + ".bin")
    put("retention.txt", namelist("inretn_type", vana_type=6, vann_type=6, resi_type=6)
        + namelist("inretn_path", in_vapath="alpha.bin", in_vnpath="n.bin", in_repath="resi.bin"))
    put("parameter.txt", namelist("inparm_type", pakx_type=6, paky_type=6, pakz_type=6, pass_type=6, pats_type=6)
        + namelist("inparm_path", in_kxpath="ksx.bin", in_kypath="ksy.bin", in_kzpath="ksz.bin",
                   in_sspath="ss.bin", in_tspath="ths.bin"))
    field3d(np.asarray(ph["head0"], dtype=np.float64), SNOVAL).astype("<f8").tofile(J("init_head.bin"))
    files.append("init_head.bin")
    # calculation region
    if extra:
        reg = np.concatenate([np.full(nx * ny, -1, np.int32), np.zeros(nx * ny, np.int32),
                              np.ones(nx * ny * nz, np.int32)])
        reg.astype("<i4").tofile(J("region.bin"))
        files.append("region.bin")
        calc_reg = dict(calc_type=6, calcreg_neib=-1, calcreg_name="region.bin", inact_name="", clas_file="")
    else:
        calc_reg = dict(calc_type=0, calcreg_neib=-1, calcreg_name="", inact_name="", clas_file="")
    # time series: rain (mm/h, records with their end time in hours) and the sea head
    tt = dict(seal_type=-1, rech_type=-1, well_type=-1, weks_type=-1, weke_type=-1, rive_type=-1, lake_type=-1,
              prec_type=-1, evap_type=-1)
    tp = dict(seal_path="", rech_path="", well_path="", weks_path="", weke_path="", rive_path="", lake_path="",
              prec_path="", evap_path="")
    tu = dict(seal_unit="", rech_unit="", well_unit="", prec_unit="", evap_unit="")
    if ph.get("rain_mm_h", 0.0) and ph.get("rain_hours", 0.0):
        with open(J("rain.bin"), "wb") as f:
            for t_end, v in ((ph["rain_hours"], ph["rain_mm_h"]), (1.0e30, 0.0)):
                np.array([t_end], dtype="<f4").tofile(f)
                np.full(nx * ny, v, dtype="<f4").tofile(f)
        files.append("rain.bin")
        tt["rech_type"], tp["rech_path"], tu["rech_unit"] = 4, "rain.bin", "HOU"
    if extra:
        sea = np.full(nx * ny * nzd, SNOVAL, dtype=np.float64)
        sea[nx * ny: 2 * nx * ny] = ph["sea_head"]
        _r4(J("sea_level.bin"), sea)
        files.append("sea_level.bin")
        tt["seal_type"], tp["seal_path"] = 6, "sea_level.bin"
    put("timeseries.txt", namelist("tinp_type", **tt) + namelist("tinp_path", **tp) + namelist("tinp_unit", **tu))
    # msg123.main
    sim_type = int(prm.get("sim_type", 0))
    if end_time is None:
        end_time = prm["end_time"] if prm.get("end_time", 1.0e30) < 1.0e29 else p.nsteps * prm["max_step"]
    if sim_type == 1:
        end = datetime.datetime(*_SDATE) + datetime.timedelta(seconds=int(round(end_time)))
        tm = dict(stime_type=0, sdate=list(_SDATE), edate=[end.year, end.month, end.day, end.hour, end.minute,
                                                          end.second], end_time=0.0, calc_unit="SEC")
    else:
        tm = dict(stime_type=0, sdate=[0] * 6, edate=[0] * 6, end_time=float(end_time), calc_unit="SEC")
    crit = float(prm["criteria"])
    if prm.get("criteria_rel", 0):
        crit = crit * float(np.max(np.abs(ph["head0"])))
    sol = dict(init_step=float(prm["ini_step"]), incr_multi=float(prm["inc_fact"]), max_step=float(prm["max_step"]),
               maxout_iter=int(prm["maxout_iter"]), criteria=crit, maxinn_iter=int(prm["maxinn_iter"]),
               precon_type=int(prm["precon_type"]))
    text = (namelist("set_simulation", sim_type=sim_type, sim_name=sim_name)
            + namelist("set_calc_time", **tm)
            + namelist("set_calc_reg", **calc_reg)
            + namelist("set_solution", **sol))
    if sol["precon_type"] == 1:
        text += namelist("set_amg", amg_nlevel=int(prm["amg_nlevel"]), maxvcy_iter=1, max_sweep=int(prm["amg_sweeps"]),
                         jac_omega=float(prm["jac_omega"]), amg_theta=float(prm["amg_theta"]))
    text += (namelist("set_grid", gridx=nx, gridy=ny, gridz=nzd, grid_type=7, grid_file="grid.txt")
             + namelist("set_retn_parm", retn_type=0, parm_type=0, retn_file="retention.txt",
                        parm_file="parameter.txt")
             + namelist("set_init", init_type=6, init_file="init_head.bin", init_dept=0.0, init_unit="")
             + namelist("set_time_input", time_input_file="timeseries.txt")
             + namelist("set_geog", geog_type=-1, geog_file="")
             + namelist("set_wtab", wtab_type=7 if "wtab" in outputs else -1)
             + namelist("set_mass", mass_type=7 if "mass" in outputs else -1, mass_file="")
             + namelist("set_out_vari", out_list=",".join(outputs))
             + namelist("set_out_unit", **{f"{v}_unit": "HOU" for v in _OUTV})
             + namelist("set_out_time", **{f"{v}_time": int(out_hours) for v in _OUTV}))
    put("msg123.main", text)
    return files


_OUTV = ("head", "rest", "srat", "wtab", "mass", "velc", "rivr", "lakr", "sufr", "dunr", "seal", "well", "rech")


# ---------------------------------------------------------------------------------------
# Reading a whole deck back into a problem
# ---------------------------------------------------------------------------------------
def _read_r4(path, n):
    a = np.fromfile(path, dtype="<f4")
    if a.size != n:
        raise ValueError(f"{path}: {a.size} values, expected {n}")
    return a


def read_deck(directory):
    """A problem (config.Problem, nondimensional like the generators) from a deck of the
    kind write_deck produces: type-7 grid; whole-grid region, or an int32 region file of
    layers (-1 inactive, 0 sea, 1 soil) with the sea layer directly above the soil; retention
    and parameter compile files naming 3D float32 fields (in_type 6); initial heads as a 3D
    float64 field (init_type 6); rain as 2D float32 records in mm/h with their end times
    (rech_type 4) and a constant 3D float32 sea level (seal_type 6).  Scaling as the
    reference applies it: alpha and Ss times len_scal, Ks times 1/len_scal in real(SP)
    (Assign_calculation.f90:117,259-260); heads times 1/len_scal in real(DP)
    (Assign_calculation.f90:471-473); sea heads real(SP) times 1/len_scal
    (Assign_boundary.f90:155); elevations from the grid's real(SP) corner and width, then
    times 1/len_scal in real(DP) (Read_input.f90:548-583, :1108-1110)."""
    import os
    from .config import Problem, default_params
    J = lambda name: os.path.join(directory, name)
    groups = read_namelists(open(J("msg123.main")).read())
    prm = solver_params(groups)
    g = groups["set_grid"]
    nx, ny, nzd = int(g["gridx"]), int(g["gridy"]), int(g["gridz"])
    if int(g.get("grid_type", -1)) != 7:
        raise ValueError("only grid_type 7 (corner and width per axis) is read here")
    lines = [l.split() for l in open(J(g["grid_file"])).read().splitlines() if l.strip()]
    (xc, xw), (yc, yw), (zc, zw) = [(F32(float(a)), F32(float(b))) for a, b, *_ in lines[1:4]]
    zs_m = np.array([zc + zw * F32(k) for k in range(nzd + 1)], dtype=F32)      # real(SP) node elevations
    ls = len_scale(float(np.max(np.abs(zs_m.astype(np.float64)))))
    lsi = F32(1.0) / ls
    nxy = nx * ny
    # region: whole grid, or layers of -1 (inactive), 0 (sea) and 1 (soil)
    reg = groups["set_calc_reg"]
    ct = int(reg.get("calc_type", -1))
    if ct == 0:
        flags = np.ones(nzd, np.int32)
    elif ct == 6:
        r = np.fromfile(J(reg["calcreg_name"]), dtype="<i4")
        if r.size != nxy * nzd:
            raise ValueError("region file size")
        r = r.reshape(nzd, nxy)
        if not all(np.all(r[k] == r[k, 0]) for k in range(nzd)):
            raise ValueError("only layered regions are read here")
        flags = r[:, 0]
    else:
        raise ValueError(f"calc_type {ct} is not read here")
    soil = np.nonzero(flags > 0)[0]
    k0, nz = int(soil[0]), len(soil)
    if not np.array_equal(soil, np.arange(k0, k0 + nz)) or np.any(flags[k0 + nz:] != 1):
        raise ValueError("the soil layers must be contiguous down to the bottom")
    sea_top = int(k0 > 0 and flags[k0 - 1] == 0)
    N = nxy * nz
    sl = slice(k0 * nxy, (k0 + nz) * nxy)
    # fields
    rp = read_namelists(open(J(groups["set_retn_parm"]["retn_file"])).read())
    pp = read_namelists(open(J(groups["set_retn_parm"]["parm_file"])).read())
    for grp, keys in ((rp["inretn_type"], ("vana_type", "vann_type", "resi_type")),
                      (pp["inparm_type"], ("pakx_type", "paky_type", "pakz_type", "pass_type", "pats_type"))):
        if any(int(grp[k]) != 6 for k in keys):
            raise ValueError("only 3D float32 fields (in_type 6) are read here")
    path = lambda grp, k: J(grp[k])
    f = {k: _read_r4(path(rp["inretn_path"], v), nxy * nzd)[sl]
         for k, v in (("alpha", "in_vapath"), ("n", "in_vnpath"), ("resi", "in_repath"))}
    f.update({k: _read_r4(path(pp["inparm_path"], v), nxy * nzd)[sl]
              for k, v in (("ksx", "in_kxpath"), ("ksy", "in_kypath"), ("ksz", "in_kzpath"), ("ss", "in_sspath"),
                           ("ths", "in_tspath"))})
    ini = groups["set_init"]
    if int(ini["init_type"]) != 6 or str(ini.get("init_unit", "")).strip():
        raise ValueError("only an initial head file of in_type 6 without a time header is read here")
    h_m = np.fromfile(J(ini["init_file"]), dtype="<f8")[sl]
    # time series
    ts = read_namelists(open(J(groups["set_time_input"]["time_input_file"])).read())
    tt, tp, tu = ts["tinp_type"], ts["tinp_path"], ts.get("tinp_unit", {})
    rain, rain_h = 0.0, 0.0
    if int(tt.get("rech_type", -1)) > 0:
        if int(tt["rech_type"]) != 4 or str(tu.get("rech_unit", "")).strip().upper() != "HOU":
            raise ValueError("only rain as 2D float32 records with hourly end times is read here")
        recs = np.fromfile(J(tp["rech_path"]), dtype="<f4").reshape(-1, nxy + 1)
        if recs.shape[0] != 2 or np.any(recs[1, 1:] != 0) or np.any(recs[0, 1:] != recs[0, 1]):
            raise ValueError("only a uniform rain followed by none is read here")
        rain, rain_h = float(recs[0, 1]), float(recs[0, 0])
    sea_head = None
    if int(tt.get("seal_type", -1)) > 0:
        if int(tt["seal_type"]) != 6 or not sea_top:
            raise ValueError("only a constant 3D sea level over a sea layer is read here")
        sv = _read_r4(J(tp["seal_path"]), nxy * nzd).reshape(nzd, nxy)[k0 - 1]
        if np.any(sv != sv[0]):
            raise ValueError("only a uniform sea level is read here")
        sea_head = float(sv[0])
    # geometry (uniform widths; elevations as the reference forms them)
    z = zs_m.astype(np.float64) * float(lsi)
    dxs = float(np.float64(F32(abs(xw))) * float(lsi))
    dys = float(np.float64(F32(abs(yw))) * float(lsi))
    top = np.repeat(z[k0:k0 + nz], nxy)
    bot = np.repeat(z[k0 + 1:k0 + nz + 1], nxy)
    hz = top - bot
    dis = np.empty((6, N))
    area = np.empty((6, N))
    dis[0] = hz * 0.5; dis[5] = hz * 0.5
    dis[1] = dys * 0.5; dis[4] = dys * 0.5
    dis[2] = dxs * 0.5; dis[3] = dxs * 0.5
    area[0] = dxs * dys; area[5] = dxs * dys
    area[1] = dxs * hz; area[4] = dxs * hz
    area[2] = dys * hz; area[3] = dys * hz
    surf = top[:nxy].copy()
    sc = lambda a, m: (np.asarray(a, F32) * (ls if m else lsi)).astype(F32)
    rate = float(F32(rain * 1.0e-3 / 3600.0) * lsi)
    prm = default_params(**dict(prm, len_scal=float(ls), criteria_rel=0, lin_tol=0.0))
    sea = np.full(nxy, float(F32(sea_head) * lsi)) if sea_head is not None else np.zeros(nxy)
    phys = dict(dx=float(abs(xw)), dy=float(abs(yw)), dz=float(abs(zw)), z_top=float(zs_m[k0]),
                alpha=f["alpha"], n=f["n"], resi=f["resi"], ths=f["ths"], ss=f["ss"], ksx=f["ksx"], ksy=f["ksy"],
                ksz=f["ksz"], head0=h_m, rain_mm_h=rain, rain_hours=rain_h, sea_head=sea_head)
    return Problem("deck", nx, ny, nz, sea_top, 0, sc(f["alpha"], True), f["n"].astype(F32), f["resi"].astype(F32),
                   f["ths"].astype(F32), sc(f["ss"], True), sc(f["ksx"], False), sc(f["ksy"], False),
                   sc(f["ksz"], False), top, dxs * dys * hz, dis.reshape(-1).copy(), area.reshape(-1).copy(),
                   np.full(nxy, dxs * dys), surf, surf.copy(), np.zeros(nxy), np.zeros(nxy), sea,
                   h_m * float(lsi), rate * np.full(nxy, dxs * dys), rain_h * 3600.0 if rain_h else 1.0e30, 0.0,
                   0, prm, phys=phys)
