"""Benchmark: simulated cell-timesteps per second of the Newton-Krylov Richards solver.

One step is one accepted implicit time step (calc_numsol: Jacobian assembly, AMG
setup, BiCGStab, line search) over the whole grid.  The workload is the
512x512x96 heterogeneous block (25,165,824 cells, sigma_lnK = 1.5, rain 20 mm/h,
adaptive steps from 600 s, Newton tolerance 1e-8 relative head), synthetic and seeded.

W warm-up steps run on the value path; every arm below then starts from that same saved
time level (msg_gpu_copy_state) and covers the same window:

* value        : mixed precision + learned initial guess (FP32/BF16 V-cycle, FP64 Krylov
                 and Newton, AMG hierarchy rebuilt every 12 time steps, CNN guess with
                 extrapolation fallback, line-search slope from BiCGStab's residual);
                 cells x K accepted steps / device time (CUDA events on the library
                 stream).  It ends at simulated time T.
* arms         : the same window up to T with one change at a time -- mixed precision
                 with the plain extrapolation (no network), FP64 with the extrapolation
                 and the same AMG reuse, and plain FP64 (the reference's method on the
                 GPU: AMG rebuilt at every Newton iteration, Newton from the previous
                 head), each with Newton/Krylov counts, rejections and simulated seconds.
                 The head and the stored water volume of the value path are compared with
                 the plain FP64 method run from the same state on the value path's own time
                 steps and solved to Newton criteria 1e-11 (the converged answer of the same
                 discrete equations).  Every arm reports its device time per step by phase.
* e2e          : the value path over the same K steps through the public C ABI with the
                 state in pinned host memory (set_state / advance / get_state each step,
                 copies inside the timed region, host wall clock).
* cpu_baseline : the C restatement of the reference path (OpenMP, all host cores) with
                 the reference's own method (AMG preconditioner as the reference applies it,
                 i.e. the level-1 DILU; FP64; previous-head start) on the 256x256x64
                 heterogeneous block's first accepted steps; the GPU runs the same method on
                 the same steps beside it.  --impl reference prints that CPU run as its line.

Run: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (torchrun): every rank solves its own seeded realisation (independent
replicas, no data-path collective); value = sum of cells x steps / max time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-timesteps/s at 1e-8 rel head tol"
# The dominant kernel pair of the value path is the assembly (k_cell<true> with both van
# Genuchten evaluations + k_flux_asm): once per Newton iteration, and it also serves as the
# line search's residual evaluation.  DRAM bytes per cell from one ncu capture of each
# (dram__bytes_read.sum + dram__bytes_write.sum): k_cell<1,0,1> 93.8 B on the 320x320x96
# block, k_flux_asm 170.8 B on the 256x256x64 block; traffic grows in proportion to the cells.
ROOF_KERNEL = 2
TRAFFIC_PER_CELL = 93.8 + 170.8
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of k_cell<1,0,1> (320x320x96 block, "
                  "93.8 B per cell) + k_flux_asm (256x256x64 block, 170.8 B per cell), scaled by cells")
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}

# Algorithmic bytes per cell of the kernels timed by msg_gpu_kernel_time (compulsory
# HBM traffic, neighbour reads cache-reused):
#  0 SpMV FP64 DIA : d 8 + six off-diagonals 48 + x 8 + y 8
#  1 calc_func     : vG pass (h, top, 5 params 20, h_old, S_old, vol -> S, kr, sto) 84
#                    + flux pass (h, kr, hy 24, ab 24, sto -> F) 80
#  2 make_matvec   : vG pair pass (h, top, params 20, h_old, S_old, vol -> S, kr, kr_per,
#                    sto, stod) 100 + assembly pass (h, kr, kr_per, hy, ab, sto, stod ->
#                    rhs, dmat, six lu, FP32 images 28) 180
ALG_BYTES = {0: 72.0, 1: 164.0, 2: 280.0}
KERNEL_NAMES = {0: "stencil SpMV (FP64, DIA)", 1: "calc_func (vG pass + flux pass)",
                2: "make_matvec (vG pair + Jacobian assembly)"}


def vcycle_bytes(sizes, sweeps, coarse_max):
    """Algorithmic bytes of one mixed-precision V-cycle (FP32 vectors, FP32 fine-level DIA
    operator, BF16 coarse off-diagonals with int32 columns, FP32 transfer weights, FP64
    dense coarsest inverse), from the level sizes [(rows, off-diagonal entries, prolongation
    entries from the level above)], level 0 = fine grid.  Every array a kernel touches is
    counted once per kernel; gathered vectors are counted once.
      fine sweep        : b 4 + x 4 + d 4 + six off-diagonals 24 + out 4 = 40 B per cell
                          (first sweep: b 8 in, d 4, x 4 and b 4 out; last: FP64 out, +4)
      residual          : like a sweep
      coarse sweep/res. : rowptr 4 + diagonal 4 + b 4 + x 4 + out 4 per row, col 4 + value 2
                          per entry (first sweep: b, d, out = 12 per row)
      restriction       : rowptr 4 per coarse row, col 4 + weight 4 per entry, fine r 4 per
                          fine row, out 4 per coarse row; prolongation the same from the
                          fine side plus the read-modify-write of x (8 per fine row)
      coarsest inverse  : 8 n^2 + 8 n"""
    sw = max(int(sweeps), 0)
    total = 0.0
    nl = len(sizes)
    for lv, (n, nnz, _) in enumerate(sizes):
        last = lv == nl - 1
        if lv > 0 and last and n <= coarse_max:
            total += 8.0 * n * n + 8.0 * n
            break
        if lv == 0:
            sweep, res = 40.0 * n, 40.0 * n
            first = 20.0 * n if sw else 16.0 * n
            final = 4.0 * n if sw else 12.0 * n          # FP64 output of the last sweep / copy
        else:
            sweep = res = 20.0 * n + 6.0 * nnz
            first = 12.0 * n if sw else 4.0 * n
            final = 0.0
        total += first + max(sw - 1, 0) * sweep + sw * sweep + final
        if not last:
            nc, _, pnnz = sizes[lv + 1]
            total += res
            total += 4.0 * nc + 8.0 * pnnz + 4.0 * n + 4.0 * nc     # restriction
            total += 4.0 * n + 8.0 * pnnz + 4.0 * nc + 8.0 * n      # prolongation
    return total


# Learned-guess CNN, algorithmic FLOPs per cell: 27 taps x 2 x (7 inputs x 16 + 16 x 16 +
# 16 x 16 + 16 x 1 output) = 34,560.  The tensor cores compute every layer with 16 input and
# 16 output channels (the zero-padded ones included): 55,296 issued FLOPs per cell.
CNN_FLOP_PER_CELL = 27 * 2 * (7 * 16 + 16 * 16 + 16 * 16 + 16 * 1)
CNN_FLOP_ISSUED_PER_CELL = 4 * 27 * 16 * 16 * 2


def _peak_value(v):
    """A peak given as a number, or as a record holding it under "value"."""
    if isinstance(v, dict):
        v = v.get("value")
    return float(v)


def load_peaks(path=None):
    """(HBM GB/s, bf16 TFLOP/s, source) from MEASURED_PEAKS.json, else the fallback figures
    measured earlier on this hardware; an unreadable file falls back too and says so."""
    p = path or os.path.join(ROOT, "MEASURED_PEAKS.json")
    if not os.path.exists(p):
        return PEAKS_FALLBACK["hbm_gbs"], PEAKS_FALLBACK["bf16_tflops"], "fallback"
    try:
        with open(p) as f:
            d = json.load(f)
        return _peak_value(d["hbm_gbs"]), _peak_value(d.get("bf16_tflops", PEAKS_FALLBACK["bf16_tflops"])), "measured"
    except (OSError, ValueError, TypeError, KeyError):
        return PEAKS_FALLBACK["hbm_gbs"], PEAKS_FALLBACK["bf16_tflops"], "fallback (measured peaks file unreadable)"


class ClockSampler:
    """SM clocks, power and clock-event reasons sampled every 200 ms during the timed region,
    the fields nvidia-smi's clocks query reports, read through NVML in this process by a
    thread of the sampler; nvidia-smi itself when NVML cannot be loaded.  NVML is
    initialised when the sampler is made -- before the warm-up, not inside the timed region:
    initialising it (as every nvidia-smi call does) can take the driver seconds on some
    machines and held up the solver's own CUDA calls when it happened in the timed window."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None
        self.nv = self.h = None
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.h = nv.nvmlDeviceGetHandleByIndex(index)
            self.nv = nv
        except Exception:
            self.nv = None

    def close(self):
        if self.nv is not None:
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass
            self.nv = None

    def _nvml_sample(self, nv, h):
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        flag = lambda bit: "Active" if r & bit else "Not Active"
        return [str(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                str(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)),
                "%.2f" % (nv.nvmlDeviceGetPowerUsage(h) / 1000.0),
                flag(nv.nvmlClocksEventReasonHwSlowdown), flag(nv.nvmlClocksEventReasonHwThermalSlowdown),
                flag(nv.nvmlClocksEventReasonSwThermalSlowdown), flag(nv.nvmlClocksEventReasonSwPowerCap)]

    def _run(self):
        nv, h = self.nv, self.h
        if nv is not None:
            while not self._stop.is_set():
                try:
                    self.samples.append(self._nvml_sample(nv, h))
                except Exception:
                    pass
                self._stop.wait(0.2)
            return
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        num = lambda v: v.replace(".", "", 1).isdigit()
        sm = [float(s[0]) for s in self.samples if num(s[0])]
        mx = [float(s[1]) for s in self.samples if num(s[1])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 3 + k and s[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, None
    import datetime
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    backend = "nccl" if torch.cuda.is_available() else "gloo"   # gloo: the CPU tests of this path
    if backend == "nccl":
        torch.cuda.set_device(local)
    # short enough that ranks left waiting for a failed one end with an error soon; the
    # longest gap between two collectives (field generation, context build) is seconds
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=180))
    return rank, ws, dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def reduce(dist, v, op):
    """MAX or SUM of a host scalar over the ranks (NCCL on the GPUs; gloo in the CPU tests)."""
    if dist is None:
        return v
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def make_problem(args, rank):
    from msg123_b200.config import make_config
    kw = {"seed": 2024 + rank}
    if args.shape:
        kw["shape"] = tuple(int(v) for v in args.shape.split("x"))
    return make_config(args.workload, **kw)


# value path: mixed precision, learned guess used directly (a failed solve from it is redone
# from the plain extrapolation), AMG hierarchy kept for 12 time steps (over a whole
# 10,000-s event at 25.2M cells: 12.2 s of device time against 12.7 s at 8 steps and 13.0 s
# at 4, with 1206 / 1202 / 1238 Newton and 1329 / 1355 / 1327 BiCGStab iterations), two-pow
# Mualem kr, line-search slope from BiCGStab's residual
FAST = dict(precision=1, amg_lag=12, guess_mode=2, guess_select=0, vg_form=1, jv_mode=1)
# one change at a time from the value path, over the same window
ARMS = (("mixed_extrapolation", dict(FAST, guess_mode=1)),
        ("fp64_extrapolation", dict(FAST, precision=0, guess_mode=1)),
        ("plain_fp64", dict(precision=0, amg_lag=0, guess_mode=0, vg_form=0)))
# the reference's own method: its AMG preconditioner as it acts (the level-1 DILU solve),
# FP64, the reference's four-pow kr, Newton from the previous head
REF_METHOD = dict(precon_type=1, ref_quirks=1, precision=0, amg_lag=0, guess_mode=0, vg_form=0)
CPU_WORKLOAD = ("hetero", (256, 256, 64))
CPU_STEPS = 4


def workload_config(args, prob):
    prm = prob.params
    return {"workload": f"{args.workload} {prob.nx}x{prob.ny}x{prob.nz} ({prob.ncalc} cells), heterogeneous "
                        f"lnKs field, 20 mm/h rain, adaptive dt from {prm['ini_step']:.0f} s",
            "solver": "Newton (Eisenstat-Walker, cubic line search) + BiCGStab + smoothed-aggregation AMG",
            "value_path": "mixed precision (FP32 V-cycle, BF16 coarse operators, FP64 Krylov/Newton/coarse LU) + "
                          "learned initial guess (guess_select %d), AMG hierarchy rebuilt every %d time steps, "
                          "two-pow form of Mualem kr (vg_form %d), line-search slope from BiCGStab's residual "
                          "(jv_mode %d)" % (FAST["guess_select"], FAST["amg_lag"], FAST["vg_form"], FAST["jv_mode"]),
            "window": f"steps {args.warmup + 1}..{args.warmup + args.steps} after {args.warmup} warm-up steps of "
                      "the value path; every arm starts from the same saved time level",
            "newton_tol": "max|dh| <= 1e-8 max|h|",
            "l2": "inputs larger than L2 (126 MB); no flush needed",
            "parallelism": f"replicas x{args.gpus}",
            **({"overrides": dict(kv.split("=", 1) for kv in args.set)} if args.set else {})}


def arm_stats(prob, st, ms, dist, fallbacks=None, timers=None):
    """Whole-job figures of one arm: value, counts per accepted step, simulated time, and the
    device time per accepted step of each phase the library times (assembly with the AMG
    rebuilds, Krylov, AMG rebuilds alone, residual evaluations)."""
    acc = max(st["accepted"], 1)
    tmax = reduce(dist, ms, "max")
    out = {"value": reduce(dist, float(prob.ncalc * st["accepted"]), "sum") / (tmax * 1e-3),
           "ms_per_step": tmax / acc, "accepted": st["accepted"], "rejected": st["rejected"],
           "newton_per_step": st["newton_total"] / acc, "krylov_per_step": st["krylov_total"] / acc,
           "backtracks": st["back_total"], "simulated_s": st["current_t"],
           "simulated_s_per_s": None}
    if fallbacks is not None:
        out["guess_fallbacks"], out["guess_rejected"] = fallbacks
    if timers is not None:
        out["phase_ms_per_step"] = {k[:-3]: round(timers[k] / acc, 3)
                                    for k in ("assembly_ms", "krylov_ms", "amg_setup_ms", "residual_ms")}
    return out


def water_volume(g, head):
    """Stored water of a state, sum over cells of vol * (theta_s S + alpha_ss S h) -- the
    quantity whose change calc_mass books as storage (Calc_function.f90:176-210)."""
    p = g.prob
    srat, _, sstor = g.srat_rperm(head)
    return float(np.sum(p.cell_vol * (p.poro.astype(np.float64) * srat + sstor * srat * head)))


def inflow_volume(prob, t0, t1):
    """Recharge volume entering between simulated times t0 and t1 (rain until rech_until)."""
    ru = prob.rech_until
    wet = max(min(t1, ru) - min(t0, ru), 0.0)
    dry = max(t1 - max(t0, ru), 0.0)
    return float(np.sum(prob.rech)) * (wet + prob.rech_after * dry)


def prep_arm(prob, kw, src, cnn, end_time=None):
    """A fresh context with settings kw, started from src's time level (the network
    attached when kw asks for the learned guess)."""
    from msg123_b200.solver import GpuSolver
    extra = {} if end_time is None else {"end_time": end_time}
    g = GpuSolver(prob, **kw, **extra)
    if kw.get("guess_mode") == 2:
        cnn.attach(g)
    g.copy_state_from(src)
    return g


class nvtx_range:
    """An NVTX range around a region (visible to a profiler that filters on it, e.g.
    ncu --nvtx --nvtx-include value_window/); a no-op where no NVTX runtime is loaded."""

    def __init__(self, name):
        self.name = name

    def __enter__(self):
        try:
            import torch
            torch.cuda.nvtx.range_push(self.name)
            self.ok = True
        except Exception:
            self.ok = False
        return self

    def __exit__(self, *a):
        if self.ok:
            import torch
            torch.cuda.nvtx.range_pop()


def run_arm_steps(g, steps):
    """run_arm one accepted step per call: the same work, timed per step (device time of
    each step from the library's events; the sum is the arm's time), so that where a slow
    window loses its time shows in the line."""
    acc = {"accepted": 0, "rejected": 0, "newton_total": 0, "krylov_total": 0, "back_total": 0}
    tm_sum = {"assembly_ms": 0.0, "krylov_ms": 0.0, "amg_setup_ms": 0.0, "residual_ms": 0.0, "total_ms": 0.0}
    step_ms, st = [], None
    while acc["accepted"] < steps:
        rc, st = g.advance(nsteps=1)
        tm = g.timers()
        for k in acc:
            acc[k] += st[k]
        for k in tm_sum:
            tm_sum[k] += tm[k]
        step_ms.append(round(tm["total_ms"], 2))
        if rc != 0 or st["accepted"] == 0:
            break
    out = dict(st, **acc)
    return out, tm_sum["total_ms"], (g.guess_fallbacks(), g.guess_rejected()), tm_sum, step_ms


def run_arm(g, steps):
    """Advance by `steps` accepted steps (or to the context's end time): (stats, device ms,
    (learned guesses redone from the extrapolation, learned guesses not used), the library's
    per-phase device times)."""
    rc, st = g.advance(nsteps=steps)
    tm = g.timers()
    return st, tm["total_ms"], (g.guess_fallbacks(), g.guess_rejected()), tm


def cpu_hw():
    """CPU model, logical CPUs and the OpenMP thread count of this host."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count(), "omp_num_threads": int(os.environ.get("OMP_NUM_THREADS", "0"))}


def cpu_run(prob, budget_s, max_steps, keep_state=False):
    """Oracle (C restatement, OpenMP, all host cores) with the reference's method, bounded in
    time: accepted steps from the initial state until max_steps or the budget."""
    from oracle.oracle import Oracle
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    threads = int(os.environ["OMP_NUM_THREADS"])
    o = Oracle(prob, **REF_METHOD)
    o.init_state()
    steps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s and steps < max_steps:
        rc, st = o.advance(nsteps=1)
        if rc != 0:
            break
        steps += 1
    dt = time.perf_counter() - t0
    head = o.get_state()["head_new"] if keep_state else None
    o.close()
    return prob.ncalc * max(steps, 1) / dt, steps, dt, threads, head


def cpu_sample_problem(args):
    from msg123_b200.config import make_config
    name, shape = CPU_WORKLOAD
    if args.cpu_shape:
        shape = tuple(int(v) for v in args.cpu_shape.split("x"))
    return make_config(name, shape=shape, seed=2024)


def cpu_sample_text(prob, steps, dt, threads):
    return (f"first {steps} accepted step(s) of the {prob.nx}x{prob.ny}x{prob.nz} heterogeneous block "
            f"(seed 2024, hydrostatic start, dt from 600 s) with the reference's method (AMG preconditioner "
            f"as the reference applies it = level-1 DILU, FP64, Newton from the previous head), C restatement "
            f"oracle/msg123_oracle.c, OpenMP {threads} threads, {dt:.1f} s")


def run_reference(args):
    rank, ws, dist = dist_setup()
    if rank == 0:
        prob = cpu_sample_problem(args)
        val, steps, dt, threads, _ = cpu_run(prob, budget_s=150.0, max_steps=min(max(1, args.steps), CPU_STEPS))
        cfg = {"workload": f"hetero {prob.nx}x{prob.ny}x{prob.nz} ({prob.ncalc} cells), heterogeneous lnKs "
                           "field, 20 mm/h rain, adaptive dt from 600 s",
               "path": "the reference's method (FP64, AMG preconditioner as applied by the reference, "
                       "previous-head start) on the host cores",
               "why_not_the_gpu_workload": "one step of the 25.2M-cell block takes about a minute on the host "
                                           "cores; the 256x256x64 block's first steps are the planned sample",
               **cpu_hw()}
        line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "cell-timesteps/s", "n_gpus": ws,
                "steps": steps, "warmup": 0, "ms_per_step": 1e3 * dt / max(steps, 1), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                "cpu_baseline": {"value": val, "unit": "cell-timesteps/s", "cores": threads, "kind": "port",
                                 "sample": cpu_sample_text(prob, steps, dt, threads)},
                "e2e": {"value": val, "unit": "cell-timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large", choices=["large", "hetero", "box"])
    ap.add_argument("--shape", default="")
    ap.add_argument("--cpu-shape", default="")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-arms", action="store_true")
    ap.add_argument("--set", action="append", default=[], metavar="KEY=VALUE",
                    help="override a solver parameter of the value path (e.g. amg_lag=8)")
    args = ap.parse_args()
    from msg123_b200.config import default_params
    for kv in args.set:
        k, v = kv.split("=", 1)
        FAST[k] = type(default_params()[k])(float(v) if "." in v or "e" in v else int(v))
    if args.impl == "reference":
        return run_reference(args)

    rank, ws, dist = dist_setup()
    from msg123_b200 import build
    if rank == 0 and build.needs_build():
        build.build()
    barrier(dist)
    from msg123_b200.learned import Cnn
    from msg123_b200.solver import GpuSolver, launch_count
    from msg123_b200.train_guess import load
    prob = make_problem(args, rank)
    cnn = load(Cnn(seed=0))
    K = args.steps

    # clock sampler (NVML) and torch (the NVTX range) set up before any timing
    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    try:
        import torch  # noqa: F401
    except Exception:
        pass

    # ---- warm-up on the value path; its time level is where every arm starts -----------
    gw = GpuSolver(prob, **FAST)
    cnn.attach(gw)
    gw.init_state()
    _, stw = gw.advance(nsteps=args.warmup)
    t_start = stw["current_t"]
    barrier(dist)

    # ---- value: mixed precision + learned guess, K accepted steps -------------------------
    ga = prep_arm(prob, FAST, gw, cnn)
    barrier(dist)
    l0 = launch_count()
    with clk, nvtx_range("value_window"):
        st, ms, fb, tm, step_ms = run_arm_steps(ga, K)
    clk.close()
    launches = launch_count() - l0
    value_arm = arm_stats(prob, st, ms, dist, fb, tm)
    value_arm["step_ms"] = step_ms
    value = value_arm["value"]
    tmax = value_arm["ms_per_step"] * max(st["accepted"], 1)
    t_end = st["current_t"]
    head_a = ga.get_state(out={"head_new": np.zeros(prob.ncalc)})["head_new"]
    vol_a = water_volume(ga, head_a)

    # kernel timings for the roofline (state of the last timed step, library stream)
    hbm, tc_peak, src = load_peaks()
    t_prec = ga.kernel_time(3, reps=5)
    vc_bytes = vcycle_bytes(ga.amg_sizes(), ga.params["amg_sweeps"], ga.params["amg_coarse_max"])
    vc_gbs = vc_bytes / (t_prec * 1e-3) / 1e9
    kt = {w: ga.kernel_time(w, reps=10) for w in (0, 1, 2)}
    gbs = {w: ALG_BYTES[w] * prob.ncalc / (kt[w] * 1e-3) / 1e9 for w in kt}
    t_setup = ga.kernel_time(4, reps=2)
    t_cnn = ga.kernel_time(5, reps=5)
    cnn_tflops = CNN_FLOP_PER_CELL * prob.ncalc / (t_cnn * 1e-3) / 1e12
    ga.close()

    # ---- the other arms over the same window (to the value path's end time T) -------------
    arms, errors = {}, None
    if not args.no_arms:
        for name, kw in ARMS:
            barrier(dist)
            g = prep_arm(prob, kw, gw, cnn, end_time=t_end)
            sta, msa, _, tma = run_arm(g, 4 * K)
            arms[name] = arm_stats(prob, sta, msa, dist, timers=tma)
            g.close()
    for a in list(arms.values()) + [value_arm]:
        a["simulated_s_per_s"] = (a["simulated_s"] - t_start) / (a["ms_per_step"] * max(a["accepted"], 1) * 1e-3)

    # ---- end to end through the public API, state in pinned host memory -------------------
    e2e = None
    if not args.no_e2e:
        import torch
        N, S = prob.ncalc, prob.ncals
        ge = prep_arm(prob, FAST, gw, cnn)
        pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
        heads = [pin(N), pin(N)]                    # [current, previous]: swapped, never copied
        sat, surf = pin(N), pin(S)
        ge.get_state(out={"head_new": heads[0], "head_old": heads[1], "srat_new": sat, "surf_head": surf})
        barrier(dist)
        acc = newton = 0
        dts = []
        t0 = time.perf_counter()
        for _ in range(K):
            ge.set_state(head_new=heads[0], head_old=heads[1], srat_old=sat, surf_head=surf)
            rc2, st2 = ge.advance(nsteps=1)
            ge.get_state(out={"head_new": heads[1], "srat_new": sat, "surf_head": surf})
            heads.reverse()
            acc += st2["accepted"]
            newton += st2["newton_total"]
            dts.append(st2["delt"])
        te = reduce(dist, time.perf_counter() - t0, "max")
        e2e = {"value": reduce(dist, float(prob.ncalc * acc), "sum") / te, "unit": "cell-timesteps/s",
               "h2d_bytes_per_step": 3 * N * 8 + S * 8, "d2h_bytes_per_step": 2 * N * 8 + S * 8,
               "accepted": acc, "newton_per_step": newton / max(acc, 1), "simulated_s": st2["current_t"],
               "same_window_as_value": bool(acc == st["accepted"] and st2["current_t"] == t_end),
               "path": "value path through msg_gpu_set_state (head_new, head_old, srat_old, surf_head) / "
                       "msg_gpu_advance / msg_gpu_get_state (head_new, srat_new, surf_head), pinned host "
                       "buffers, host wall clock"}
        ge.close()
        # ---- errors of the value path against the converged FP64 answer -----------------
        # (the reference's method from the same state, each step forced to the value path's
        # dt and solved to Newton criteria 1e-11 instead of 1e-8, so the difference is the
        # value path's own error: its arithmetic and its stopping point)
        if not args.no_arms:
            gf = GpuSolver(prob, **dict(ARMS[-1][1], sim_type=0, inc_fact=1.0, criteria=1.0e-11, maxout_iter=60))
            gf.copy_state_from(gw)
            for dt in dts:
                gf.set_state(delt=dt)
                gf.advance(nsteps=1)
            head_d = gf.get_state(out={"head_new": np.zeros(prob.ncalc)})["head_new"]
            vol_d = water_volume(gf, head_d)
            inflow = inflow_volume(prob, t_start, t_end)
            errors = {"against": "plain FP64 (reference method) solved to Newton criteria 1e-11 on the value "
                                 "path's own time steps",
                      "steps": len(dts),
                      "head_rel": reduce(dist, float(np.max(np.abs(head_a - head_d)) / np.max(np.abs(head_d))), "max"),
                      "stored_water_rel_inflow": reduce(dist, abs(vol_a - vol_d) / inflow, "max"),
                      "inflow_volume": inflow}
            gf.close()
    gw.close()

    # ---- CPU baseline: the reference's method on the host cores, and on the GPU beside it --
    cpu, refgpu = None, None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cp = cpu_sample_problem(args)
        val, steps, dt, threads, head_c = cpu_run(cp, budget_s=60.0, max_steps=CPU_STEPS, keep_state=True)
        cpu = {"value": val, "unit": "cell-timesteps/s", "cores": threads, "kind": "port",
               "sample": cpu_sample_text(cp, steps, dt, threads), **cpu_hw()}
        gr = GpuSolver(cp, **REF_METHOD)
        gr.init_state()
        rcr, str_ = gr.advance(nsteps=steps)
        head_g = gr.get_state(out={"head_new": np.zeros(cp.ncalc)})["head_new"]
        refgpu = {"workload": f"hetero {cp.nx}x{cp.ny}x{cp.nz}", "steps": str_["accepted"],
                  "value": cp.ncalc * str_["accepted"] / (gr.timers()["total_ms"] * 1e-3),
                  "newton_per_step": str_["newton_total"] / max(str_["accepted"], 1),
                  "speedup_over_cpu": cp.ncalc * str_["accepted"] / (gr.timers()["total_ms"] * 1e-3) / val,
                  "head_rel_vs_cpu": float(np.max(np.abs(head_g - head_c)) / np.max(np.abs(head_c)))}
        gr.close()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-timesteps/s", "n_gpus": ws, "steps": K,
            "warmup": args.warmup, "ms_per_step": value_arm["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 (Krylov/Newton) + f32/bf16 (V-cycle)",
            "data": "synthetic (seeded lnKs field and van Genuchten draws)", "config": workload_config(args, prob),
            "newton": {k: value_arm[k] for k in ("accepted", "rejected", "newton_per_step", "krylov_per_step",
                                                 "backtracks", "simulated_s", "guess_fallbacks", "guess_rejected")},
            "window_start_s": t_start,
            "arms": dict(arms, value=value_arm) if arms else None,
            "speedup_over_plain_fp64": (value / arms["plain_fp64"]["value"]) if arms else None,
            "errors_vs_fp64": errors,
            "roofline": {"kernel": KERNEL_NAMES[ROOF_KERNEL], "bound": "hbm", "achieved": gbs[ROOF_KERNEL],
                         "peak": hbm, "unit": "GB/s", "frac": gbs[ROOF_KERNEL] / hbm, "peak_source": src,
                         "alg_bytes_per_cell": ALG_BYTES[ROOF_KERNEL], "cells_per_launch": prob.ncalc,
                         "ms_per_launch": kt[ROOF_KERNEL], "traffic": TRAFFIC_PER_CELL * prob.ncalc,
                         "traffic_source": TRAFFIC_SOURCE,
                         "others": dict({KERNEL_NAMES[w]: {"ms": kt[w], "GB/s": gbs[w], "frac": gbs[w] / hbm}
                                         for w in (0, 1, 2) if w != ROOF_KERNEL},
                                        **{"learned-guess CNN, 4 tcgen05 convolutions": {
                                            "ms": t_cnn, "TFLOP/s": cnn_tflops, "frac": cnn_tflops / tc_peak,
                                            "bound": "tensor", "peak_TFLOP/s": tc_peak,
                                            "flop_per_cell": CNN_FLOP_PER_CELL,
                                            "issued_TFLOP/s": CNN_FLOP_ISSUED_PER_CELL * prob.ncalc / (t_cnn * 1e-3) / 1e12},
                                           "mixed V-cycle, all levels": {
                                            "ms": t_prec, "GB/s": vc_gbs, "frac": vc_gbs / hbm,
                                            "alg_bytes": vc_bytes}}),
                         "vcycle_mixed_ms": t_prec, "amg_setup_ms": t_setup},
            "cpu_baseline": cpu, "reference_method_gpu": refgpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    cnn.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
