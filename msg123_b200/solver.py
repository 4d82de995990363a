"""Host-side mirror of Msg123's solver interface over libmsg123gpu.so.

``GpuSolver`` exposes the reference routines under their reference names:

* ``calc_func(h)``            -- Calc_function.f90:24-101
* ``srat_rperm(h, pertur)``   -- Calc_parameter.f90:15-77
* ``make_matvec()``           -- Make_linearsystem.f90:24-68
* ``solve_linalg(...)``       -- Linear_solution.f90:26-58
* ``calc_numsol()``           -- Nonlinear_solution.f90:33-294
* ``advance(nsteps)``         -- Msg.f90:83-104 with Time_module.f90:34-273
* ``calc_mass()``             -- Calc_function.f90:103-174

Every call goes through the C ABI declared in include/msg123_gpu.h.  There is no
CPU fallback: if the CUDA library is missing or no GPU is present the
constructor raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi
from .abi import dptr, iptr

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmsg123gpu.so")
_lib = None


class MsgError(RuntimeError):
    pass


def load_library():
    """Load libmsg123gpu.so (built in-tree by msg123_b200/build.py) or raise."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise MsgError(f"{LIB_PATH} is missing: run `python -m msg123_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.msg_gpu_last_error.restype = C.c_char_p
    L.msg_gpu_create.argtypes = [C.POINTER(abi.MsgGrid), C.POINTER(abi.MsgParams), C.POINTER(vp)]
    L.msg_gpu_destroy.argtypes = [vp]
    L.msg_gpu_destroy.restype = None
    L.msg_gpu_get_connect.argtypes = [vp, abi.PI, abi.PI, abi.PI, abi.PI, abi.PI, abi.PD, abi.PD, abi.PI]
    L.msg_gpu_init_state.argtypes = [vp, abi.PD, C.c_double]
    L.msg_gpu_set_state.argtypes = [vp, abi.PD, abi.PD, abi.PD, abi.PD, C.c_double]
    L.msg_gpu_get_state.argtypes = [vp, abi.PD, abi.PD, abi.PD, abi.PD, abi.PD]
    L.msg_gpu_set_recharge.argtypes = [vp, abi.PD]
    L.msg_gpu_srat_rperm.argtypes = [vp, abi.PD, C.c_double, abi.PD, abi.PD, abi.PD]
    L.msg_gpu_calc_func.argtypes = [vp, abi.PD, abi.PD]
    L.msg_gpu_make_matvec.argtypes = [vp, abi.PD, abi.PD, abi.PD]
    L.msg_gpu_set_system.argtypes = [vp, abi.PD, abi.PD, abi.PD]
    L.msg_gpu_precond.argtypes = [vp, abi.PD, abi.PD]
    L.msg_gpu_vecjacf.argtypes = [vp, abi.PD, abi.PD, abi.PD]
    L.msg_gpu_solve_linalg.argtypes = [vp, C.c_double, C.c_double, abi.PD, abi.PD, abi.PI, abi.PI]
    L.msg_gpu_calc_numsol.argtypes = [vp, C.POINTER(abi.MsgStats)]
    L.msg_gpu_advance.argtypes = [vp, C.c_int32, C.c_double, C.c_double, C.POINTER(abi.MsgRunStats)]
    L.msg_gpu_calc_mass.argtypes = [vp, abi.PD]
    L.msg_gpu_timers.argtypes = [vp, abi.PD]
    L.msg_gpu_set_timing.argtypes = [vp, C.c_int32]
    L.msg_gpu_kernel_time.argtypes = [vp, C.c_int32, C.c_int32, abi.PD]
    L.msg_gpu_set_tuning.argtypes = [vp, C.c_int32, C.c_int32]
    L.msg_gpu_amg_nlevel.argtypes = [vp]
    L.msg_gpu_amg_level_sizes.argtypes = [vp, C.c_int32, abi.PI, abi.PI, abi.PI]
    L.msg_gpu_amg_level.argtypes = [vp, C.c_int32, abi.PI, abi.PI, abi.PD, abi.PD, abi.PI, abi.PI, abi.PD, abi.PI]
    L.msg_gpu_dense_inverse.argtypes = [C.c_int32, abi.PD, abi.PD]
    L.msg_gpu_launch_count.restype = C.c_longlong
    L.msg_gpu_launch_count.argtypes = []
    _lib = L
    return L


def launch_count():
    return int(load_library().msg_gpu_launch_count())


def dense_inverse(a):
    """Inverse of a dense square matrix (the AMG coarsest-level solve) on the GPU."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    inv = np.zeros((n, n))
    _check(load_library().msg_gpu_dense_inverse(n, dptr(a), dptr(inv)), "dense_inverse")
    return inv


def read_restart(path, ncalc, len_scal):
    """(heads, time) from a restart file of the reference (host code, no GPU)."""
    L = load_library()
    L.msg_gpu_read_restart.argtypes = [C.c_char_p, C.c_int32, C.c_double, abi.PD, abi.PD]
    h = np.zeros(int(ncalc))
    t = np.zeros(1)
    _check(L.msg_gpu_read_restart(os.fsencode(path), int(ncalc), C.c_double(len_scal), dptr(h), dptr(t)),
           "read_restart")
    return h, float(t[0])


def _check(rc, what):
    if rc < 0:
        msg = load_library().msg_gpu_last_error().decode(errors="replace")
        raise MsgError(f"{what} failed ({abi.STATUS_NAMES.get(rc, rc)}): {msg}")
    return rc


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class GpuSolver:
    """One solver context on the current CUDA device for a config.Problem."""

    def __init__(self, prob, **overrides):
        L = load_library()
        self.prob = prob
        prm = dict(prob.params)
        prm.update(overrides)
        self.params = prm
        self._g = abi.fill_grid(prob)
        self._p = abi.fill_params(prm)
        h = C.c_void_p()
        _check(L.msg_gpu_create(C.byref(self._g), C.byref(self._p), C.byref(h)), "msg_gpu_create")
        self.h = h
        self.n = prob.ncalc
        self.ncals = prob.ncals
        nnz = C.c_int32()
        _check(L.msg_gpu_get_connect(self.h, None, None, None, None, None, None, None, C.byref(nnz)), "get_connect")
        self.nnz = nnz.value
        self.set_recharge(prob.rech)

    def close(self):
        if getattr(self, "h", None):
            load_library().msg_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- topology ---------------------------------------------------------------------
    def connect(self):
        N, M = self.n, self.nnz
        out = dict(offind=np.zeros(N + 1, np.int32), offrow=np.zeros(M, np.int32), conn_dir=np.zeros(M, np.int32),
                   left_off=np.zeros(M, np.int32), right_off=np.zeros(M, np.int32),
                   hydf=np.zeros(M), abyd=np.zeros(M))
        _check(load_library().msg_gpu_get_connect(self.h, iptr(out["offind"]), iptr(out["offrow"]),
                                                  iptr(out["conn_dir"]), iptr(out["left_off"]),
                                                  iptr(out["right_off"]), dptr(out["hydf"]), dptr(out["abyd"]),
                                                  None), "get_connect")
        return out

    # -- state --------------------------------------------------------------------------
    def init_state(self, head=None, delt=None):
        head = self.prob.head0 if head is None else head
        delt = self.params["ini_step"] if delt is None else delt
        _check(load_library().msg_gpu_init_state(self.h, dptr(_f64(head)), C.c_double(delt)), "init_state")

    def set_state(self, head_new=None, head_old=None, srat_old=None, surf_head=None, delt=0.0):
        arrs = [None if a is None else _f64(a) for a in (head_new, head_old, srat_old, surf_head)]
        _check(load_library().msg_gpu_set_state(self.h, *(dptr(a) for a in arrs), C.c_double(delt)), "set_state")

    def get_state(self, out=None):
        """Copy the state to host arrays: new float64 arrays of all five fields, or the
        fields named in `out` (C-contiguous float64 arrays, e.g. views of pinned memory);
        fields missing from `out` are not copied."""
        N, S = self.n, self.ncals
        sizes = (("head_new", N), ("head_old", N), ("srat_new", N), ("srat_old", N), ("surf_head", S))
        if out is None:
            out = {k: np.zeros(n) for k, n in sizes}
        for k, n in sizes:
            a = out.get(k)
            if a is not None and (a.dtype != np.float64 or not a.flags.c_contiguous or a.size != n):
                raise ValueError(f"get_state: {k} must be a C-contiguous float64 array of {n}")
        _check(load_library().msg_gpu_get_state(self.h, *(dptr(out.get(k)) for k, _ in sizes)), "get_state")
        return out

    def copy_state_from(self, other):
        """Take the whole time level of another context of the same grid (msg_gpu_copy_state)."""
        L = load_library()
        L.msg_gpu_copy_state.argtypes = [C.c_void_p, C.c_void_p]
        _check(L.msg_gpu_copy_state(self.h, other.h), "copy_state")

    def water_table(self):
        """calc_wtable of the current state (Calc_output.f90:20-52): [ncals] heads,
        nondimensional like head_new."""
        L = load_library()
        L.msg_gpu_water_table.argtypes = [C.c_void_p, abi.PD]
        out = np.zeros(self.ncals)
        _check(L.msg_gpu_water_table(self.h, dptr(out)), "water_table")
        return out

    def set_convlog(self, on=True):
        """Record every Newton iteration (the reference's convergence-log line)."""
        L = load_library()
        L.msg_gpu_set_convlog.argtypes = [C.c_void_p, C.c_int32]
        _check(L.msg_gpu_set_convlog(self.h, 1 if on else 0), "set_convlog")

    def convlog(self):
        """Recorded iterations since the last call, oldest first (list of dicts); see
        msg123_b200.convlog for writing them in the reference's format."""
        L = load_library()
        L.msg_gpu_convlog.argtypes = [C.c_void_p, C.POINTER(abi.MsgConvRec), C.c_int32]
        out = []
        buf = (abi.MsgConvRec * 4096)()
        while True:
            k = _check(L.msg_gpu_convlog(self.h, buf, 4096), "convlog")
            out.extend(buf[i].as_dict() for i in range(k))
            if k < 4096:
                return out

    def guess_fallbacks(self):
        """Learned guesses whose Newton run failed and was redone from the extrapolation."""
        L = load_library()
        L.msg_gpu_guess_fallbacks.argtypes = [C.c_void_p]
        return int(L.msg_gpu_guess_fallbacks(self.h))

    def guess_rejected(self):
        """Learned guesses not used because their residual exceeded the extrapolation's."""
        L = load_library()
        L.msg_gpu_guess_rejected.argtypes = [C.c_void_p]
        return int(L.msg_gpu_guess_rejected(self.h))

    def write_restart(self, path):
        """Restart file of the reference (gfortran records: time, head * len_scal)."""
        L = load_library()
        L.msg_gpu_write_restart.argtypes = [C.c_void_p, C.c_char_p]
        _check(L.msg_gpu_write_restart(self.h, os.fsencode(path)), "write_restart")

    def set_wells(self, well_index, well_conn, abyd, bott, rate):
        """Well table (msg_gpu_set_wells): well_index [nwell+1] prefix offsets, well_conn
        1-based cells, abyd_well per connection; well_bott and pumping rate per well."""
        L = load_library()
        L.msg_gpu_set_wells.argtypes = [C.c_void_p, C.c_int32, abi.PI, abi.PI, abi.PD, abi.PD, abi.PD]
        wi = np.ascontiguousarray(well_index, dtype=np.int32)
        arrs = (np.ascontiguousarray(well_conn, np.int32), _f64(abyd), _f64(bott), _f64(rate))
        _check(L.msg_gpu_set_wells(self.h, len(wi) - 1, iptr(wi), iptr(arrs[0]), dptr(arrs[1]), dptr(arrs[2]),
                                   dptr(arrs[3])), "set_wells")

    def set_rivers(self, cells, head, bott, abyd):
        """River cells (msg_gpu_set_rivers): 1-based surface cells, stage, bed, area/distance."""
        self._stage("msg_gpu_set_rivers", cells, head, bott, abyd)

    def set_lakes(self, cells, head, bott, abyd):
        """Lake cells (msg_gpu_set_lakes): 1-based surface cells, stage, bed, area/distance."""
        self._stage("msg_gpu_set_lakes", cells, head, bott, abyd)

    def _stage(self, name, cells, head, bott, abyd):
        fn = getattr(load_library(), name)
        fn.argtypes = [C.c_void_p, C.c_int32, abi.PI, abi.PD, abi.PD, abi.PD]
        c = np.ascontiguousarray(cells, dtype=np.int32)
        _check(fn(self.h, len(c), iptr(c), dptr(_f64(head)), dptr(_f64(bott)), dptr(_f64(abyd))), name)

    def set_recharge(self, rech):
        _check(load_library().msg_gpu_set_recharge(self.h, dptr(_f64(rech))), "set_recharge")

    # -- reference routines -----------------------------------------------------------------
    def srat_rperm(self, pres, pertur=0.0):
        N = self.n
        s, k, ss = np.zeros(N), np.zeros(N), np.zeros(N)
        _check(load_library().msg_gpu_srat_rperm(self.h, dptr(_f64(pres)), C.c_double(pertur), dptr(s), dptr(k),
                                                 dptr(ss)), "srat_rperm")
        return s, k, ss

    def calc_func(self, x):
        f = np.zeros(self.n)
        _check(load_library().msg_gpu_calc_func(self.h, dptr(_f64(x)), dptr(f)), "calc_func")
        return f

    def make_matvec(self):
        d, lu, r = np.zeros(self.n), np.zeros(self.nnz), np.zeros(self.n)
        _check(load_library().msg_gpu_make_matvec(self.h, dptr(d), dptr(lu), dptr(r)), "make_matvec")
        return d, lu, r

    def set_system(self, dmat, lumat, rhs):
        _check(load_library().msg_gpu_set_system(self.h, dptr(_f64(dmat)), dptr(_f64(lumat)), dptr(_f64(rhs))),
               "set_system")

    def precond(self, r):
        z = np.zeros(self.n)
        _check(load_library().msg_gpu_precond(self.h, dptr(_f64(r)), dptr(z)), "precond")
        return z

    def vecjacf(self, x, v):
        out = np.zeros(self.n)
        _check(load_library().msg_gpu_vecjacf(self.h, dptr(_f64(x)), dptr(_f64(v)), dptr(out)), "vecjacf")
        return out

    def solve_linalg(self, init_norm, errtol, x0=None):
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        last = C.c_double()
        it = C.c_int32()
        conv = C.c_int32()
        _check(load_library().msg_gpu_solve_linalg(self.h, C.c_double(init_norm), C.c_double(errtol), dptr(x),
                                                   C.byref(last), C.byref(it), C.byref(conv)), "solve_linalg")
        return x, last.value, it.value, conv.value

    def calc_numsol(self):
        st = abi.MsgStats()
        rc = _check(load_library().msg_gpu_calc_numsol(self.h, C.byref(st)), "calc_numsol")
        return rc, st.as_dict()

    def advance(self, nsteps=None, rech_until=None, rech_after=None):
        nsteps = self.prob.nsteps if nsteps is None else nsteps
        ru = self.prob.rech_until if rech_until is None else rech_until
        ra = self.prob.rech_after if rech_after is None else rech_after
        rs = abi.MsgRunStats()
        rc = _check(load_library().msg_gpu_advance(self.h, int(nsteps), C.c_double(ru), C.c_double(ra), C.byref(rs)),
                    "advance")
        return rc, rs.as_dict()

    def calc_mass(self):
        out = np.zeros(9)
        _check(load_library().msg_gpu_calc_mass(self.h, dptr(out)), "calc_mass")
        return out

    def cell_mass(self):
        """calc_cell_mas (Calc_output.f90:54-91): the step's volumes per cell, dict of sto,
        con, sea, wel [ncalc] and rec, sur, riv, lak, drn [ncals]."""
        L = load_library()
        L.msg_gpu_cell_mass.argtypes = [C.c_void_p] + [abi.PD] * 9
        N, S = self.n, self.ncals
        keys = (("sto", N), ("con", N), ("sea", N), ("wel", N), ("rec", S), ("sur", S), ("riv", S), ("lak", S),
                ("drn", S))
        out = {k: np.zeros(n) for k, n in keys}
        _check(L.msg_gpu_cell_mass(self.h, *(dptr(out[k]) for k, _ in keys)), "cell_mass")
        return out

    def velocity(self):
        """calc_outvelc (Calc_output.f90:168-241) at head_new: (facev [6, ncalc] face-major,
        pointv [3, ncalc] x, y, z)."""
        L = load_library()
        L.msg_gpu_velocity.argtypes = [C.c_void_p, abi.PD, abi.PD]
        fv, pv = np.zeros(6 * self.n), np.zeros(3 * self.n)
        _check(L.msg_gpu_velocity(self.h, dptr(fv), dptr(pv)), "velocity")
        return fv.reshape(6, self.n), pv.reshape(3, self.n)

    def amg_sizes(self):
        """(rows, off-diagonal entries, prolongation entries from the level above) of each
        level of the last AMG setup, level 0 = Jacobian (its prolongation count is 0)."""
        L = load_library()
        out = []
        for lv in range(L.msg_gpu_amg_nlevel(self.h)):
            n, nnz, pnnz = C.c_int32(), C.c_int32(), C.c_int32()
            _check(L.msg_gpu_amg_level_sizes(self.h, lv, C.byref(n), C.byref(nnz), C.byref(pnnz)), "amg sizes")
            out.append((n.value, nnz.value, pnnz.value if lv > 0 else 0))
        return out

    def amg_levels(self):
        """The AMG hierarchy of the last setup (level 0 = Jacobian), as numpy arrays."""
        L = load_library()
        levels = []
        for lv in range(L.msg_gpu_amg_nlevel(self.h)):
            n, nnz, pnnz = C.c_int32(), C.c_int32(), C.c_int32()
            _check(L.msg_gpu_amg_level_sizes(self.h, lv, C.byref(n), C.byref(nnz), C.byref(pnnz)), "amg sizes")
            n, nnz, pnnz = n.value, nnz.value, pnnz.value
            d = dict(n=n, offind=np.zeros(n + 1, np.int32), offrow=np.zeros(max(nnz, 1), np.int32)[:nnz],
                     dmat=np.zeros(n), lumat=np.zeros(max(nnz, 1))[:nnz])
            args = [None, None, None, None]
            if lv > 0:
                nf = levels[-1]["n"]
                d.update(pindex=np.zeros(nf + 1, np.int32), poffrow=np.zeros(max(pnnz, 1), np.int32)[:pnnz],
                         pval=np.zeros(max(pnnz, 1))[:pnnz], agg=np.zeros(nf, np.int32))
                args = [iptr(d["pindex"]), iptr(d["poffrow"]), dptr(d["pval"]), iptr(d["agg"])]
            _check(L.msg_gpu_amg_level(self.h, lv, iptr(d["offind"]), iptr(d["offrow"]), dptr(d["dmat"]),
                                       dptr(d["lumat"]), *args), "amg level")
            levels.append(d)
        return levels

    def set_timing(self, on=True):
        _check(load_library().msg_gpu_set_timing(self.h, int(bool(on))), "set_timing")

    def set_tuning(self, blk_cell, blk_smooth):
        _check(load_library().msg_gpu_set_tuning(self.h, int(blk_cell), int(blk_smooth)), "set_tuning")

    def kernel_time(self, which, reps=20):
        ms = C.c_double()
        _check(load_library().msg_gpu_kernel_time(self.h, int(which), int(reps), C.byref(ms)), "kernel_time")
        return ms.value

    def timers(self):
        out = np.zeros(5)
        _check(load_library().msg_gpu_timers(self.h, dptr(out)), "timers")
        return dict(zip(("assembly_ms", "krylov_ms", "amg_setup_ms", "residual_ms", "total_ms"), out.tolist()))
