"""Learned Newton initial guess: training driver over the CUDA kernels in
msg123_b200/csrc/msg_learned.cu.

The network predicts the correction to the linear extrapolation of the head
(h0 = h_t + r (h_t - h_{t-1}) + s * CNN(features)); it is trained on time steps the
GPU solver itself produces and plugged into the Newton time loop with
guess_mode = 2 (the plain extrapolation is the fallback when a Newton solve fails).
"""
import ctypes as C

import numpy as np

from . import abi
from .solver import GpuSolver, load_library, _check

NCH = 16
NTAP = 27
NLAYER = 4


def _lib():
    L = load_library()
    if not getattr(L, "_cnn_ready", False):
        vp = C.c_void_p
        L.msg_gpu_cnn_create.argtypes = [C.c_int32, C.POINTER(vp)]
        L.msg_gpu_cnn_destroy.argtypes = [vp]
        L.msg_gpu_cnn_destroy.restype = None
        L.msg_gpu_cnn_nparam.argtypes = []
        L.msg_gpu_cnn_set_deadband.argtypes = [vp, C.c_float]
        L.msg_gpu_cnn_get_weights.argtypes = [vp, abi.PF]
        L.msg_gpu_cnn_set_weights.argtypes = [vp, abi.PF]
        L.msg_gpu_cnn_collect.argtypes = [vp, vp]
        L.msg_gpu_cnn_nsamples.argtypes = [vp]
        L.msg_gpu_cnn_set_capacity.argtypes = [vp, C.c_int32, C.c_int32]
        L.msg_gpu_cnn_seen.argtypes = [vp]
        L.msg_gpu_cnn_seen.restype = C.c_longlong
        L.msg_gpu_cnn_add_sample.argtypes = [vp, C.c_int32, C.c_int32, C.c_int32, abi.PF, abi.PF]
        L.msg_gpu_cnn_loss_grad.argtypes = [vp, C.c_int32, abi.PD, abi.PF, abi.PF]
        L.msg_gpu_cnn_infer.argtypes = [vp, C.c_int32, abi.PF]
        L.msg_gpu_cnn_infer_withhold.argtypes = [vp, C.c_int32, C.c_int32, abi.PF]
        L.msg_gpu_cnn_train.argtypes = [vp, C.c_int32, C.c_float, C.c_float, C.c_int32, abi.PD]
        L.msg_gpu_cnn_attach.argtypes = [vp, vp]
        L.msg_gpu_guess_fallbacks.argtypes = [vp]
        L.msg_gpu_guess_rejected.argtypes = [vp]
        L._cnn_ready = True
    return L


class Cnn:
    """Network handle: weights, optimizer state and a device-resident sample set."""

    def __init__(self, seed=0):
        h = C.c_void_p()
        _check(_lib().msg_gpu_cnn_create(int(seed), C.byref(h)), "cnn_create")
        self.h = h
        self.nparam = _lib().msg_gpu_cnn_nparam()

    def close(self):
        if getattr(self, "h", None):
            _lib().msg_gpu_cnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_deadband(self, dead):
        _check(_lib().msg_gpu_cnn_set_deadband(self.h, C.c_float(dead)), "cnn_set_deadband")

    def get_weights(self):
        w = np.zeros(self.nparam, np.float32)
        _check(_lib().msg_gpu_cnn_get_weights(self.h, abi.fptr(w)), "cnn_get_weights")
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(_lib().msg_gpu_cnn_set_weights(self.h, abi.fptr(w)), "cnn_set_weights")

    def collect(self, solver):
        _check(_lib().msg_gpu_cnn_collect(self.h, solver.h), "cnn_collect")

    def nsamples(self):
        return _lib().msg_gpu_cnn_nsamples(self.h)

    def set_capacity(self, cap, seed=0):
        """Keep at most `cap` samples, a uniform (reservoir) sample of every step collected."""
        _check(_lib().msg_gpu_cnn_set_capacity(self.h, int(cap), int(seed)), "cnn_set_capacity")

    def seen(self):
        """Steps offered to collect() since the capacity was set."""
        return int(_lib().msg_gpu_cnn_seen(self.h))

    def add_sample(self, shape, x, y):
        nx, ny, nz = shape
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        _check(_lib().msg_gpu_cnn_add_sample(self.h, nx, ny, nz, abi.fptr(x), abi.fptr(y)), "cnn_add_sample")

    def loss_grad(self, sample=0, want_grad=True, want_out=False, n=None):
        loss = C.c_double()
        g = np.zeros(self.nparam, np.float32) if want_grad else None
        o = np.zeros(n, np.float32) if want_out else None
        _check(_lib().msg_gpu_cnn_loss_grad(self.h, int(sample), C.byref(loss), abi.fptr(g), abi.fptr(o)),
               "cnn_loss_grad")
        return loss.value, g, o

    def infer(self, sample, n):
        """Output of the tensor-core (tcgen05) inference path on stored sample `sample`."""
        o = np.zeros(n, np.float32)
        _check(_lib().msg_gpu_cnn_infer(self.h, int(sample), abi.fptr(o)), "cnn_infer")
        return o

    def infer_withhold(self, sample, n, tile):
        """Test hook: inference with the input box of `tile` never loaded.  Returns the
        library status (MSG_ERR_CUDA expected) and the error message."""
        o = np.zeros(n, np.float32)
        rc = _lib().msg_gpu_cnn_infer_withhold(self.h, int(sample), int(tile), abi.fptr(o))
        return rc, load_library().msg_gpu_last_error().decode()

    def train(self, iters, lr=1e-3, weight_decay=1e-4, seed=0):
        loss = C.c_double()
        _check(_lib().msg_gpu_cnn_train(self.h, int(iters), C.c_float(lr), C.c_float(weight_decay), int(seed),
                                        C.byref(loss)), "cnn_train")
        return loss.value

    def attach(self, solver):
        _check(_lib().msg_gpu_cnn_attach(solver.h, self.h), "cnn_attach")

    def detach(self, solver):
        """The solver stops using the network (guess_mode 2 falls back to extrapolation)."""
        _check(_lib().msg_gpu_cnn_attach(solver.h, None), "cnn_attach")


def unpack(w):
    """Flat parameter vector -> list of (W[27,16,16] (tap, co, ci), b[16]) per layer."""
    per = NTAP * NCH * NCH + NCH
    out = []
    for l in range(NLAYER):
        blk = w[l * per:(l + 1) * per]
        out.append((blk[:NTAP * NCH * NCH].reshape(NTAP, NCH, NCH), blk[NTAP * NCH * NCH:]))
    return out


def generate(cnn, problems, steps_per_problem, warmup=2, **solver_kw):
    """Run the GPU solver (plain extrapolation guess) on each problem and store every
    accepted step as a training sample.  Returns the number of samples added."""
    n0 = cnn.nsamples()
    for p in problems:
        kw = dict(guess_mode=1)
        kw.update(solver_kw)
        with GpuSolver(p, **kw) as g:
            g.init_state()
            g.advance(nsteps=warmup)
            for _ in range(steps_per_problem):
                rc, st = g.advance(nsteps=1)
                if rc != 0 or st["accepted"] != 1:
                    break
                cnn.collect(g)
    return cnn.nsamples() - n0


def newton_per_step(problem, steps, cnn=None, guess_mode=1, warmup=2, **solver_kw):
    """Newton iterations per accepted step (and fallbacks) with a given guess mode."""
    with GpuSolver(problem, guess_mode=guess_mode, **solver_kw) as g:
        if cnn is not None:
            cnn.attach(g)
        g.init_state()
        g.advance(nsteps=warmup)
        rc, st = g.advance(nsteps=steps)
        fb = (_lib().msg_gpu_guess_fallbacks(g.h), _lib().msg_gpu_guess_rejected(g.h))
        if cnn is not None:
            _lib().msg_gpu_cnn_attach(g.h, None)
    return st["newton_total"] / max(st["accepted"], 1), st, fb
