"""Batched ensemble of independent realisations (uneven grid sizes and Newton counts).

Members are drawn as in msg123_b200.config.make_member (nx, ny in 64..160, nz in
32..48, sigma_lnK in 0.5..1.5) and advanced together by msg_gpu_ensemble_advance:
worker threads take members from a shared queue and drive each on its own CUDA
stream, so the GPU overlaps the members' kernels.  The worker count and the launch
shapes come from the autotuner.
"""
import ctypes as C
import time

import numpy as np

from . import abi
from .autotune import tune
from .config import make_member
from .solver import GpuSolver, load_library, _check

ENSEMBLE = dict(precision=1, amg_lag=4, guess_mode=1)


def _lib():
    L = load_library()
    if not getattr(L, "_ens_ready", False):
        L.msg_gpu_ensemble_advance.argtypes = [C.POINTER(C.c_void_p), C.c_int32, C.c_int32, abi.PD, abi.PD,
                                               C.c_int32, C.POINTER(abi.MsgRunStats)]
        L.msg_gpu_set_tuning.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
        L._ens_ready = True
    return L


class Ensemble:
    def __init__(self, nmembers=64, seed0=0, seeds=None, **overrides):
        """Members seed0 .. seed0 + nmembers - 1, or the explicit member `seeds` (a rank's share)."""
        kw = dict(ENSEMBLE)
        kw.update(overrides)
        self.seeds = list(seeds) if seeds is not None else [seed0 + k for k in range(nmembers)]
        nmembers = len(self.seeds)
        self.members = []
        for k in self.seeds:
            p = make_member(k)
            g = GpuSolver(p, **kw)
            p.dis2face = p.face_area = None      # only needed while the context is created
            self.members.append(g)
        self.cells = np.array([g.n for g in self.members], dtype=np.int64)
        self._ptrs = (C.c_void_p * nmembers)(*[g.h.value for g in self.members])
        self._ru = np.array([g.prob.rech_until for g in self.members], dtype=np.float64)
        self._ra = np.array([g.prob.rech_after for g in self.members], dtype=np.float64)
        self.workers = 16

    def close(self):
        for g in self.members:
            g.close()
        self.members = []

    def init_state(self):
        for g in self.members:
            g.init_state()

    def advance(self, nsteps, workers=None):
        n = len(self.members)
        st = (abi.MsgRunStats * n)()
        w = workers or self.workers
        t0 = time.perf_counter()
        rc = _lib().msg_gpu_ensemble_advance(self._ptrs, n, int(nsteps), abi.dptr(self._ru), abi.dptr(self._ra),
                                             int(w), st)
        dt = time.perf_counter() - t0
        _check(rc, "ensemble_advance")
        stats = [s.as_dict() for s in st]
        return dt, stats

    def autotune(self, worker_candidates=(8, 16, 32, 64), probe_steps=1):
        """Launch shapes from a median-size member, then the worker count by timing.  The
        members advance by the probe steps (the first one assembles the systems whose
        kernels are timed)."""
        med = self.members[int(np.argsort(self.cells)[len(self.cells) // 2])]
        self.advance(probe_steps)
        bc, bs, _ = tune(med)
        for g in self.members:
            _lib().msg_gpu_set_tuning(g.h, bc, bs)
        best, best_rate = None, -1.0
        for w in worker_candidates:
            dt, stats = self.advance(probe_steps, workers=w)
            rate = float(sum(c * s["accepted"] for c, s in zip(self.cells, stats))) / dt
            if rate > best_rate:
                best, best_rate = w, rate
        self.workers = best
        return {"blk_cell": bc, "blk_smooth": bs, "workers": best}

    def throughput(self, nsteps):
        dt, stats = self.advance(nsteps)
        cells_steps = float(sum(c * s["accepted"] for c, s in zip(self.cells, stats)))
        newton = [s["newton_total"] / max(s["accepted"], 1) for s in stats]
        return cells_steps / dt, dt, stats, newton
