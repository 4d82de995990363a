"""ctypes wrapper of the CPU oracle (oracle/msg123_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the msg123_b200 package.  The methods
mirror the reference routines the C file restates (calc_func, make_matvec,
solve_linalg, calc_numsol, the time loop, calc_mass).
"""
import ctypes as C
import os
import subprocess

import numpy as np

from msg123_b200 import abi
from msg123_b200.abi import dptr, iptr

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(os.path.join(_HERE, "msg123_oracle.c")):
            build()
        L = C.CDLL(_LIB)
        vp = C.c_void_p
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(abi.MsgGrid), C.POINTER(abi.MsgParams)]
        L.orc_destroy.argtypes = [vp]
        for f in ("orc_nnz", "orc_nseal", "orc_amg_nlevel"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = C.c_int
        L.orc_counter.argtypes = [vp, C.c_int]
        L.orc_counter.restype = C.c_longlong
        for f in ("orc_calc_numsol",):
            getattr(L, f).restype = C.c_int
        L.orc_advance.restype = C.c_int
        L.orc_advance.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.POINTER(abi.MsgRunStats)]
        L.orc_calc_numsol.argtypes = [vp, C.POINTER(abi.MsgStats)]
        L.orc_solve_linalg.restype = C.c_int
        L.orc_solve_linalg.argtypes = [vp, C.c_double, C.c_double, abi.PD, abi.PD, abi.PI]
        L.orc_init_state.argtypes = [vp, abi.PD, C.c_double]
        L.orc_set_state.argtypes = [vp, abi.PD, abi.PD, abi.PD, abi.PD, C.c_double]
        L.orc_srat_rperm.argtypes = [vp, abi.PD, C.c_double, abi.PD, abi.PD, abi.PD]
        L.orc_cell_mass.argtypes = [vp] + [abi.PD] * 9
        L.orc_set_wells.argtypes = [vp, C.c_int, abi.PI, abi.PI, abi.PD, abi.PD, abi.PD]
        L.orc_set_rivers.argtypes = [vp, C.c_int, abi.PI, abi.PD, abi.PD, abi.PD]
        L.orc_set_lakes.argtypes = [vp, C.c_int, abi.PI, abi.PD, abi.PD, abi.PD]
        L.orc_velocity.argtypes = [vp, abi.PD, abi.PD]
        L.orc_amg_level_sizes.argtypes = [vp, C.c_int, abi.PI, abi.PI, abi.PI]
        L.orc_amg_level.argtypes = [vp, C.c_int, abi.PI, abi.PI, abi.PD, abi.PD, abi.PI, abi.PI, abi.PD, abi.PI]
        L.orc_set_aggregation.argtypes = [vp, C.c_int]
        _lib = L
    return _lib


def dense_inverse(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    inv = np.zeros((n, n))
    lib().orc_dense_inverse(C.c_int(n), dptr(a), dptr(inv))
    return inv


class Oracle:
    """CPU oracle instance for one Problem (msg123_b200.config.Problem)."""

    def __init__(self, prob, **overrides):
        self.prob = prob
        prm = dict(prob.params)
        prm.update(overrides)
        self.params = prm
        self._g = abi.fill_grid(prob)
        self._p = abi.fill_params(prm)
        self.h = lib().orc_create(C.byref(self._g), C.byref(self._p))
        self.n = prob.ncalc
        self.ncals = prob.ncals
        self.nnz = lib().orc_nnz(self.h)
        lib().orc_set_recharge(C.c_void_p(self.h), dptr(np.ascontiguousarray(prob.rech, dtype=np.float64)))

    def close(self):
        if self.h:
            lib().orc_destroy(C.c_void_p(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- connectivity ---------------------------------------------------------------
    def connect(self):
        N, M = self.n, self.nnz
        out = dict(offind=np.zeros(N + 1, np.int32), offrow=np.zeros(M, np.int32), conn_dir=np.zeros(M, np.int32),
                   left_off=np.zeros(M, np.int32), right_off=np.zeros(M, np.int32),
                   hydf=np.zeros(M), abyd=np.zeros(M))
        lib().orc_get_connect(C.c_void_p(self.h), iptr(out["offind"]), iptr(out["offrow"]), iptr(out["conn_dir"]),
                              iptr(out["left_off"]), iptr(out["right_off"]), dptr(out["hydf"]), dptr(out["abyd"]))
        return out

    # -- state ----------------------------------------------------------------------
    def init_state(self, head=None, delt=None):
        head = self.prob.head0 if head is None else head
        delt = self.params["ini_step"] if delt is None else delt
        lib().orc_init_state(C.c_void_p(self.h), dptr(np.ascontiguousarray(head, dtype=np.float64)), C.c_double(delt))

    def set_state(self, head_new=None, head_old=None, srat_old=None, surf_head=None, delt=0.0):
        c = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        hn, ho, so, sh = c(head_new), c(head_old), c(srat_old), c(surf_head)
        lib().orc_set_state(C.c_void_p(self.h), dptr(hn), dptr(ho), dptr(so), dptr(sh), C.c_double(delt))

    def get_state(self):
        N, S = self.n, self.ncals
        out = dict(head_new=np.zeros(N), head_old=np.zeros(N), srat_new=np.zeros(N), srat_old=np.zeros(N),
                   surf_head=np.zeros(S))
        lib().orc_get_state(C.c_void_p(self.h), *(dptr(out[k]) for k in ("head_new", "head_old", "srat_new", "srat_old", "surf_head")))
        return out

    def set_recharge(self, rech):
        lib().orc_set_recharge(C.c_void_p(self.h), dptr(np.ascontiguousarray(rech, dtype=np.float64)))

    # -- routines -------------------------------------------------------------------
    def srat_rperm(self, pres, pertur=0.0):
        N = self.n
        s, k, ss = np.zeros(N), np.zeros(N), np.zeros(N)
        lib().orc_srat_rperm(C.c_void_p(self.h), dptr(np.ascontiguousarray(pres, dtype=np.float64)),
                             C.c_double(pertur), dptr(s), dptr(k), dptr(ss))
        return s, k, ss

    def calc_func(self, x):
        f = np.zeros(self.n)
        lib().orc_calc_func(C.c_void_p(self.h), dptr(np.ascontiguousarray(x, dtype=np.float64)), dptr(f))
        return f

    def make_matvec(self):
        d, lu, r = np.zeros(self.n), np.zeros(self.nnz), np.zeros(self.n)
        lib().orc_make_matvec(C.c_void_p(self.h), dptr(d), dptr(lu), dptr(r))
        return d, lu, r

    def set_system(self, dmat, lumat, rhs):
        lib().orc_set_system(C.c_void_p(self.h), dptr(np.ascontiguousarray(dmat, dtype=np.float64)),
                             dptr(np.ascontiguousarray(lumat, dtype=np.float64)),
                             dptr(np.ascontiguousarray(rhs, dtype=np.float64)))

    def precon_dilu(self):
        d = np.zeros(self.n)
        lib().orc_precon_dilu(C.c_void_p(self.h), dptr(d))
        return d

    def solve_ilu(self, d, r):
        z = np.zeros(self.n)
        lib().orc_solve_ilu(C.c_void_p(self.h), dptr(np.ascontiguousarray(d)), dptr(np.ascontiguousarray(r)), dptr(z))
        return z

    def precond(self, r):
        z = np.zeros(self.n)
        lib().orc_precond(C.c_void_p(self.h), dptr(np.ascontiguousarray(r, dtype=np.float64)), dptr(z))
        return z

    def matvec(self, x):
        y = np.zeros(self.n)
        lib().orc_matvec(C.c_void_p(self.h), dptr(np.ascontiguousarray(x, dtype=np.float64)), dptr(y))
        return y

    def solve_linalg(self, init_norm, errtol, x0=None):
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        last = C.c_double(0.0)
        it = C.c_int32(0)
        conv = lib().orc_solve_linalg(C.c_void_p(self.h), C.c_double(init_norm), C.c_double(errtol), dptr(x),
                                      C.byref(last), C.byref(it))
        return x, last.value, it.value, conv

    def vecjacf(self, x, v):
        out = np.zeros(self.n)
        lib().orc_vecjacf(C.c_void_p(self.h), dptr(np.ascontiguousarray(x)), dptr(np.ascontiguousarray(v)), dptr(out))
        return out

    def calc_numsol(self):
        st = abi.MsgStats()
        rc = lib().orc_calc_numsol(C.c_void_p(self.h), C.byref(st))
        return rc, st.as_dict()

    def advance(self, nsteps=None, rech_until=None, rech_after=None):
        nsteps = self.prob.nsteps if nsteps is None else nsteps
        ru = self.prob.rech_until if rech_until is None else rech_until
        ra = self.prob.rech_after if rech_after is None else rech_after
        rs = abi.MsgRunStats()
        rc = lib().orc_advance(C.c_void_p(self.h), int(nsteps), C.c_double(ru), C.c_double(ra), C.byref(rs))
        return rc, rs.as_dict()

    def calc_mass(self):
        out = np.zeros(9)
        lib().orc_calc_mass(C.c_void_p(self.h), dptr(out))
        return out

    def cell_mass(self):
        """calc_cell_mas per cell: dict of sto, con, sea, wel [ncalc] and rec, sur, riv, lak, drn [ncals]."""
        N, S = self.prob.ncalc, self.prob.ncals
        keys = (("sto", N), ("con", N), ("sea", N), ("wel", N), ("rec", S), ("sur", S), ("riv", S), ("lak", S),
                ("drn", S))
        out = {k: np.zeros(n) for k, n in keys}
        lib().orc_cell_mass(C.c_void_p(self.h), *(dptr(out[k]) for k, _ in keys))
        return out

    def set_wells(self, well_index, well_conn, abyd, bott, rate):
        """Well table as set_wellconn leaves it: well_index [nwell+1] prefix offsets, well_conn
        1-based cells, abyd_well per connection; well_bott and the pumping rate read_well per well."""
        wi = np.ascontiguousarray(well_index, dtype=np.int32)
        lib().orc_set_wells(C.c_void_p(self.h), len(wi) - 1, iptr(wi), iptr(np.ascontiguousarray(well_conn, np.int32)),
                            dptr(np.ascontiguousarray(abyd, np.float64)), dptr(np.ascontiguousarray(bott, np.float64)),
                            dptr(np.ascontiguousarray(rate, np.float64)))

    def set_rivers(self, cells, head, bott, abyd):
        """River cells (rive2cals, 1-based surface cells) with stage, bed and area/distance."""
        self._stage(lib().orc_set_rivers, cells, head, bott, abyd)

    def set_lakes(self, cells, head, bott, abyd):
        """Lake cells (lake2cals, 1-based surface cells) with stage, bed and area/distance."""
        self._stage(lib().orc_set_lakes, cells, head, bott, abyd)

    def _stage(self, fn, cells, head, bott, abyd):
        c = np.ascontiguousarray(cells, np.int32)
        fn(C.c_void_p(self.h), len(c), iptr(c), *(dptr(np.ascontiguousarray(a, np.float64)) for a in (head, bott, abyd)))

    def velocity(self):
        """calc_outvelc: (facev [6, ncalc] face-major, pointv [3, ncalc] x, y, z)."""
        N = self.prob.ncalc
        fv, pv = np.zeros(6 * N), np.zeros(3 * N)
        lib().orc_velocity(C.c_void_p(self.h), dptr(fv), dptr(pv))
        return fv.reshape(6, N), pv.reshape(3, N)

    def counters(self):
        return {k: lib().orc_counter(C.c_void_p(self.h), i) for i, k in enumerate(("func", "matvec", "prec"))}

    # -- AMG inspection ---------------------------------------------------------------
    def set_aggregation(self, mode):
        """Aggregation of the next AMG setups (precon_type 1, ref_quirks 0): 0 the MIS-2 the
        CUDA library runs, 1 the priority-queue aggregation of make_aggregation
        (Make_amg_matrix.f90:113-222, :633-768), a structural comparison only."""
        lib().orc_set_aggregation(C.c_void_p(self.h), int(mode))

    def amg_levels(self):
        L = lib()
        nl = L.orc_amg_nlevel(C.c_void_p(self.h))
        levels = []
        for lv in range(nl):
            n, nnz, pnnz = C.c_int32(), C.c_int32(), C.c_int32()
            L.orc_amg_level_sizes(C.c_void_p(self.h), lv, C.byref(n), C.byref(nnz), C.byref(pnnz))
            n, nnz, pnnz = n.value, nnz.value, pnnz.value
            d = dict(n=n, offind=np.zeros(n + 1, np.int32), offrow=np.zeros(max(nnz, 1), np.int32)[:nnz],
                     dmat=np.zeros(n), lumat=np.zeros(max(nnz, 1))[:nnz])
            if lv > 0:
                nf = levels[-1]["n"]
                d.update(pindex=np.zeros(nf + 1, np.int32), poffrow=np.zeros(max(pnnz, 1), np.int32)[:pnnz],
                         pval=np.zeros(max(pnnz, 1))[:pnnz], agg=np.zeros(nf, np.int32))
                L.orc_amg_level(C.c_void_p(self.h), lv, iptr(d["offind"]), iptr(d["offrow"]), dptr(d["dmat"]),
                                dptr(d["lumat"]), iptr(d["pindex"]), iptr(d["poffrow"]), dptr(d["pval"]), iptr(d["agg"]))
            else:
                L.orc_amg_level(C.c_void_p(self.h), lv, iptr(d["offind"]), iptr(d["offrow"]), dptr(d["dmat"]),
                                dptr(d["lumat"]), None, None, None, None)
            levels.append(d)
        return levels
