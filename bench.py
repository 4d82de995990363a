"""Benchmark: simulated cell-timesteps per second of the Newton-Krylov Richards solver.

One step is one accepted implicit time step (calc_numsol: Jacobian assembly, AMG
setup, BiCGStab, line search) over the whole grid.  The workload is the
512x512x96 heterogeneous block (25,165,824 cells, sigma_lnK = 1.5, rain 20 mm/h,
adaptive steps from 600 s, Newton tolerance 1e-8 relative head), synthetic and seeded.

* value     : mixed precision + learned initial guess (FP32/BF16 V-cycle, FP64 Krylov and
              Newton, AMG hierarchy rebuilt every 4 time steps, CNN guess with extrapolation
              fallback); cells x accepted steps / device time of the K timed steps
              (CUDA events on the library stream).
* plain_fp64: the reference's method on the same field on the GPU (FP64 everywhere,
              AMG rebuilt at every Newton iteration, Newton started from the previous
              head), the path the north-star ratio is taken against.
* e2e       : the mixed+learned path through the public C ABI with the state in host
              memory (head/srat/surface copied in and out through set_state/get_state
              every step).
* cpu_baseline / --impl reference: the C restatement of the reference path (OpenMP,
              all host cores) on a bounded block of the same generator.

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
# DRAM bytes per cell of one calc_func (k_cell<false> + k_flux_res), from one ncu capture of
# the 256x256x64 block (dram__bytes_read.sum + dram__bytes_write.sum, both kernels) divided
# by its 4,194,304 cells; traffic grows in proportion to the cells.
TRAFFIC_CALC_FUNC_PER_CELL = 150.0
TRAFFIC_SOURCE = "profiles/calc_func_kernels_hetero_256x256x64.md, scaled by cells"
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


# Learned-guess CNN on the tensor cores: 4 convolutions x 27 taps x 16 x 16 (channels padded
# to 16, as the tcgen05 MMA computes them) x 2 flops per cell.
CNN_FLOP_PER_CELL = 4 * 27 * 16 * 16 * 2


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
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
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


# learned guess used directly (no residual check: it costs two residual evaluations per step
# and rarely rejects a guess in this window); a failed solve from it is redone from the
# plain extrapolation
FAST = dict(precision=1, amg_lag=4, guess_mode=2, guess_select=0, vg_form=1)
PLAIN = dict(precision=0, amg_lag=0, guess_mode=0)


def workload_config(args, prob):
    prm = prob.params
    return {"workload": f"{args.workload} {prob.nx}x{prob.ny}x{prob.nz} ({prob.ncalc} cells), heterogeneous "
                        f"lnKs field, 20 mm/h rain, adaptive dt from {prm['ini_step']:.0f} s",
            "solver": "Newton (Eisenstat-Walker, cubic line search) + BiCGStab + smoothed-aggregation AMG",
            "value_path": "mixed precision (FP32 V-cycle, BF16 coarse operators, FP64 Krylov/Newton/coarse LU) + "
                          "learned initial guess (used directly, extrapolation fallback), AMG hierarchy rebuilt every 4 "
                          "time steps, two-pow form of Mualem kr (vg_form 1)",
            "baseline_path": "plain FP64, AMG rebuilt every Newton iteration, Newton from the previous head",
            "newton_tol": "max|dh| <= 1e-8 max|h|",
            "l2": "inputs larger than L2 (126 MB); no flush needed",
            "parallelism": f"replicas x{args.gpus}",
            **({"overrides": dict(kv.split("=", 1) for kv in args.set)} if args.set else {})}


def timed_advance(g, steps):
    rc, st = g.advance(nsteps=steps)
    return st, g.timers()["total_ms"]


def cpu_run(prob, budget_s, max_steps):
    """Oracle (C restatement, OpenMP) on the plain FP64 path, bounded in time."""
    from oracle.oracle import Oracle
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    o = Oracle(prob, **PLAIN)
    o.init_state()
    steps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s and steps < max_steps:
        rc, st = o.advance(nsteps=1)
        if rc != 0:
            break
        steps += 1
    dt = time.perf_counter() - t0
    o.close()
    return prob.ncalc * max(steps, 1) / dt, steps, dt, threads


def cpu_sample_problem(args):
    from msg123_b200.config import make_config
    return make_config(args.workload, shape=tuple(int(v) for v in args.cpu_shape.split("x")), seed=2024)


def run_reference(args):
    rank, ws, dist = dist_setup()
    if rank == 0:
        prob = cpu_sample_problem(args)
        val, steps, dt, threads = cpu_run(prob, budget_s=60.0, max_steps=max(1, args.steps))
        sample = (f"{steps} accepted step(s) of a {prob.nx}x{prob.ny}x{prob.nz} block of the same generator "
                  f"(plain FP64 path), C restatement oracle/msg123_oracle.c with OpenMP, {dt:.1f} s")
        line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "cell-timesteps/s", "n_gpus": ws,
                "steps": steps, "warmup": 0, "ms_per_step": 1e3 * dt / max(steps, 1), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"{args.workload} generator, {prob.nx}x{prob.ny}x{prob.nz} block",
                           "path": "plain FP64 (reference method)"},
                "cpu_baseline": {"value": val, "unit": "cell-timesteps/s", "cores": threads, "kind": "port",
                                 "sample": sample},
                "e2e": {"value": val, "unit": "cell-timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large", choices=["large", "hetero", "box"])
    ap.add_argument("--shape", default="")
    ap.add_argument("--cpu-shape", default="96x96x96")
    ap.add_argument("--plain-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
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

    # ---- mixed precision + learned guess: the headline -------------------------------
    g = GpuSolver(prob, **FAST)
    cnn.attach(g)
    g.init_state()
    g.advance(nsteps=args.warmup)
    barrier(dist)
    l0 = launch_count()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        st, ms = timed_advance(g, args.steps)
    launches = launch_count() - l0
    tmax = reduce(dist, ms, "max")
    value = reduce(dist, float(prob.ncalc * st["accepted"]), "sum") / (tmax * 1e-3)

    # kernel timings for the roofline (state of the last timed step, library stream)
    hbm, tc_peak, src = load_peaks()
    # the V-cycle first: make_matvec below re-assembles at the converged head, whose
    # right-hand side is far smaller than any the solve passes to the preconditioner
    t_prec = g.kernel_time(3, reps=5)
    vc_bytes = vcycle_bytes(g.amg_sizes(), g.params["amg_sweeps"], g.params["amg_coarse_max"])
    vc_gbs = vc_bytes / (t_prec * 1e-3) / 1e9
    kt = {w: g.kernel_time(w, reps=10) for w in (0, 1, 2)}
    gbs = {w: ALG_BYTES[w] * prob.ncalc / (kt[w] * 1e-3) / 1e9 for w in kt}
    t_setup = g.kernel_time(4, reps=2)
    t_cnn = g.kernel_time(5, reps=5)
    cnn_tflops = CNN_FLOP_PER_CELL * prob.ncalc / (t_cnn * 1e-3) / 1e12

    # end to end through the public API, state in host memory
    e2e = None
    if not args.no_e2e:
        import torch
        N, S = prob.ncalc, prob.ncals
        # state in pinned host memory, copied in and out through the public C ABI every step
        pin = {k: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
               for k, n in (("head_new", N), ("head_old", N), ("srat_new", N), ("srat_old", N), ("surf_head", S))}
        g.get_state(out=pin)
        barrier(dist)
        t0 = time.perf_counter()
        acc = 0
        for _ in range(args.steps):
            g.set_state(head_new=pin["head_new"], head_old=pin["head_old"], srat_old=pin["srat_old"],
                        surf_head=pin["surf_head"])
            rc2, st2 = g.advance(nsteps=1)
            g.get_state(out=pin)
            pin["srat_old"][:] = pin["srat_new"]
            acc += st2["accepted"]
        te = reduce(dist, time.perf_counter() - t0, "max")
        e2e = {"value": reduce(dist, float(prob.ncalc * acc), "sum") / te, "unit": "cell-timesteps/s",
               "h2d_bytes_per_step": 3 * N * 8 + S * 8, "d2h_bytes_per_step": 4 * N * 8 + S * 8,
               "path": "mixed + learned through msg_gpu_set_state / msg_gpu_advance / msg_gpu_get_state, "
                       "pinned host buffers"}
    g.close()

    # ---- plain FP64 reference method on the same field ----------------------------------
    plain = None
    if not args.no_plain:
        gp = GpuSolver(prob, **PLAIN)
        gp.init_state()
        gp.advance(nsteps=1)
        barrier(dist)
        stp, msp = timed_advance(gp, args.plain_steps)
        tpm = reduce(dist, msp, "max")
        pv = reduce(dist, float(prob.ncalc * stp["accepted"]), "sum") / (tpm * 1e-3)
        plain = {"value": pv, "ms_per_step": tpm / max(stp["accepted"], 1),
                 "newton_per_step": stp["newton_total"] / max(stp["accepted"], 1),
                 "krylov_per_step": stp["krylov_total"] / max(stp["accepted"], 1),
                 "steps": stp["accepted"], "simulated_s_per_step": None,
                 "speedup_of_value": value / pv}
        gp.close()

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cp = cpu_sample_problem(args)
        val, steps, dt, threads = cpu_run(cp, budget_s=25.0, max_steps=args.steps)
        cpu = {"value": val, "unit": "cell-timesteps/s", "cores": threads, "kind": "port",
               "sample": f"{steps} accepted step(s) of a {cp.nx}x{cp.ny}x{cp.nz} block of the same generator on the "
                         f"plain FP64 path, C restatement oracle/msg123_oracle.c with OpenMP ({dt:.1f} s)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-timesteps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tmax / max(st["accepted"], 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 (Krylov/Newton) + f32/bf16 (V-cycle)",
            "data": "synthetic (seeded lnKs field and van Genuchten draws)", "config": workload_config(args, prob),
            "newton": {"accepted": st["accepted"], "rejected": st["rejected"],
                       "newton_per_step": st["newton_total"] / max(st["accepted"], 1),
                       "krylov_per_step": st["krylov_total"] / max(st["accepted"], 1),
                       "backtracks": st["back_total"], "simulated_s": st["current_t"]},
            "plain_fp64": plain,
            "roofline": {"kernel": KERNEL_NAMES[1], "bound": "hbm", "achieved": gbs[1], "peak": hbm,
                         "unit": "GB/s", "frac": gbs[1] / hbm, "peak_source": src,
                         "alg_bytes_per_cell": ALG_BYTES[1], "cells_per_launch": prob.ncalc,
                         "ms_per_launch": kt[1], "traffic": TRAFFIC_CALC_FUNC_PER_CELL * prob.ncalc,
                         "traffic_source": TRAFFIC_SOURCE,
                         "others": dict({KERNEL_NAMES[w]: {"ms": kt[w], "GB/s": gbs[w], "frac": gbs[w] / hbm}
                                         for w in (0, 2)},
                                        **{"learned-guess CNN, 4 tcgen05 convolutions": {
                                            "ms": t_cnn, "TFLOP/s": cnn_tflops, "frac": cnn_tflops / tc_peak,
                                            "bound": "tensor", "peak_TFLOP/s": tc_peak},
                                           "mixed V-cycle, all levels": {
                                            "ms": t_prec, "GB/s": vc_gbs, "frac": vc_gbs / hbm,
                                            "alg_bytes": vc_bytes}}),
                         "vcycle_mixed_ms": t_prec, "amg_setup_ms": t_setup},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    cnn.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
