"""ctypes mirror of include/msg123_gpu.h (structs and status codes).

The layouts here must match the C header field for field; tests/test_abi.py
checks the sizes and offsets against the compiled library.
"""
import ctypes as C

MSG_OK = 0
MSG_NEWTON_MAXIT = 1
MSG_NAN = 2
MSG_LINESEARCH_FAIL = 3
MSG_DIVERGED = 4
MSG_DT_TOO_SMALL = 5
MSG_ERR_ARG = -1
MSG_ERR_CUDA = -2
MSG_ERR_SIZE = -3
MSG_ERR_STATE = -4

STATUS_NAMES = {
    MSG_OK: "ok", MSG_NEWTON_MAXIT: "newton_maxit", MSG_NAN: "nan",
    MSG_LINESEARCH_FAIL: "linesearch_fail", MSG_DIVERGED: "diverged",
    MSG_DT_TOO_SMALL: "dt_too_small", MSG_ERR_ARG: "err_arg", MSG_ERR_CUDA: "err_cuda",
    MSG_ERR_SIZE: "err_size", MSG_ERR_STATE: "err_state",
}

PF = C.POINTER(C.c_float)
PD = C.POINTER(C.c_double)
PI = C.POINTER(C.c_int32)


class MsgGrid(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("sea_top", C.c_int32), ("free_drainage", C.c_int32), ("pad0", C.c_int32),
        ("reta", PF), ("retn", PF), ("resi", PF), ("poro", PF), ("ss", PF),
        ("ksx", PF), ("ksy", PF), ("ksz", PF),
        ("cell_top", PD), ("cell_vol", PD),
        ("dis2face", PD), ("face_area", PD),
        ("area_r", PD),
        ("surf_top", PD), ("surf_bott", PD), ("surf_reli", PD), ("surf_parm", PD),
        ("sea_head", PD),
    ]


class MsgParams(C.Structure):
    _fields_ = [
        ("len_scal", C.c_double), ("criteria", C.c_double), ("lin_tol", C.c_double),
        ("criteria_rel", C.c_int32), ("maxout_iter", C.c_int32), ("maxinn_iter", C.c_int32),
        ("precon_type", C.c_int32), ("ref_quirks", C.c_int32), ("precision", C.c_int32),
        ("amg_nlevel", C.c_int32), ("amg_coarse_max", C.c_int32), ("amg_sweeps", C.c_int32),
        ("jac_omega", C.c_float), ("amg_theta", C.c_float), ("smooth_omega", C.c_float),
        ("sim_type", C.c_int32), ("amg_lag", C.c_int32),
        ("ini_step", C.c_double), ("inc_fact", C.c_double), ("max_step", C.c_double),
        ("end_time", C.c_double), ("guess_mode", C.c_int32), ("guess_select", C.c_int32),
        ("vg_form", C.c_int32), ("jv_mode", C.c_int32),
    ]


class MsgStats(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("out_iter", C.c_int32), ("inner_total", C.c_int32),
        ("back_total", C.c_int32), ("in_iter_last", C.c_int32), ("back_iter_last", C.c_int32),
        ("maxnun", C.c_int32), ("pad", C.c_int32),
        ("maxvar", C.c_double), ("l2_new", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class MsgRunStats(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("accepted", C.c_int32), ("rejected", C.c_int32),
        ("newton_total", C.c_int32), ("krylov_total", C.c_int32), ("back_total", C.c_int32),
        ("current_t", C.c_double), ("delt", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class MsgConvRec(C.Structure):
    """One Newton iteration of the convergence log (msg_convrec_t)."""
    _fields_ = [
        ("time", C.c_double), ("delt", C.c_double),
        ("out_iter", C.c_int32), ("in_iter", C.c_int32), ("back_iter", C.c_int32), ("cell", C.c_int32),
        ("maxvar", C.c_double), ("dmat", C.c_double), ("rhs", C.c_double), ("head", C.c_double),
        ("status", C.c_int32), ("pad", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


def fptr(a):
    """float32 numpy array -> POINTER(c_float) (None passes NULL)."""
    return None if a is None else a.ctypes.data_as(PF)


def dptr(a):
    return None if a is None else a.ctypes.data_as(PD)


def iptr(a):
    return None if a is None else a.ctypes.data_as(PI)


def fill_grid(prob):
    """Build a MsgGrid from a Problem (msg123_b200.config).  The returned struct
    references the Problem's arrays, which must stay alive while it is used."""
    g = MsgGrid()
    g.nx, g.ny, g.nz = prob.nx, prob.ny, prob.nz
    g.sea_top = int(prob.sea_top)
    g.free_drainage = int(prob.free_drainage)
    for name in ("reta", "retn", "resi", "poro", "ss", "ksx", "ksy", "ksz"):
        setattr(g, name, fptr(getattr(prob, name)))
    for name in ("cell_top", "cell_vol", "dis2face", "face_area", "area_r",
                 "surf_top", "surf_bott", "surf_reli", "surf_parm", "sea_head"):
        setattr(g, name, dptr(getattr(prob, name)))
    return g


def fill_params(prm):
    p = MsgParams()
    for k, _ in MsgParams._fields_:
        if k.startswith("pad"):
            continue
        setattr(p, k, prm[k])
    return p
