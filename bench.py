"""Benchmark: simulated cell-timesteps per second of the Newton-Krylov Richards solver.

One "step" is one accepted implicit time step (calc_numsol: Jacobian assembly,
AMG/ILU setup, BiCGStab, line search) over the whole grid.  value = cells x
accepted steps / device time of the K timed steps (CUDA events on the library's
stream).  e2e = the same metric through the public C ABI with the state in host
memory: every step copies head_new / head_old / srat_old / surf_head in and
head_new / srat_new out (the way a Fortran caller of calc_numsol holds its state).

Workloads (synthetic, seeded; see msg123_b200/config.py):
  hetero : 256x256x64 heterogeneous block, plain FP64 BiCGStab + AMG (default)
  box    : 20x20x50 infiltration box, BiCGStab + ILU(0)
  large  : 512x512x96 block

Run: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU (torchrun): every rank solves its own seeded realisation; no data-path
collective exists (independent replicas), value = sum of cells x steps / max time.
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

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}

# Algorithmic bytes per cell for the kernel classes timed by msg_gpu_kernel_time
# (compulsory traffic, neighbour reads assumed cache-reused):
#  SpMV FP64 DIA: d 8 + six off-diagonals 48 + x 8 + y 8
#  calc_func    : vG pass (h 8, top 8, 5 params 20, h_old 8, S_old 8, vol 8 -> S 8, kr 8, sto 8)
#                 + flux pass (h 8, kr 8, hy 24, ab 24, sto 8 -> F 8)
#  make_matvec  : vG pair pass (inputs 60 -> S, kr, kr_per, sto, stod 40)
#                 + assembly pass (h, kr, kr_per 24, hy, ab 48, sto, stod 16 -> rhs, dmat 16, lu 48)
ALG_BYTES = {0: 72.0, 1: 84.0 + 80.0, 2: 100.0 + 152.0}
KERNEL_NAMES = {0: "stencil SpMV (FP64, DIA)", 1: "calc_func (vG + flux)", 2: "make_matvec (vG pair + assembly)"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


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
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if len(s) > 3 + k and
                          s[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def make_problem(args, rank):
    from msg123_b200.config import make_config
    kw = {}
    if args.shape:
        kw["shape"] = tuple(int(v) for v in args.shape.split("x"))
    if args.workload in ("hetero", "large"):
        kw["seed"] = 2024 + rank
    p = make_config(args.workload, **kw)
    if args.precision == "mixed":
        p.params["precision"] = 1
    if args.precon:
        p.params["precon_type"] = 0 if args.precon == "ilu" else 1
    return p


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, None
    import datetime
    import torch
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, ws, dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def allmax(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allsum(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def cpu_baseline(args, prob, budget_s=20.0):
    """The oracle (C restatement, OpenMP) on a bounded prefix of the same workload."""
    from oracle.oracle import Oracle
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    o = Oracle(prob)
    o.init_state()
    steps = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < budget_s and steps < max(1, args.steps):
        rc, st = o.advance(nsteps=1)
        if rc != 0:
            break
        steps += 1
    dt = time.perf_counter() - t0
    o.close()
    return {"value": prob.ncalc * steps / dt, "unit": "cell-timesteps/s", "cores": threads, "kind": "port",
            "sample": f"first {steps} accepted step(s) of the same {prob.nx}x{prob.ny}x{prob.nz} workload, "
                      f"C restatement (oracle/msg123_oracle.c, -O2, OpenMP) in {dt:.1f} s"}


def run_reference(args):
    rank, ws, dist = dist_setup()
    if rank != 0:
        return
    prob = make_problem(args, 0)
    from oracle.oracle import Oracle
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    o = Oracle(prob)
    o.init_state()
    for _ in range(args.warmup):
        o.advance(nsteps=1)
        break   # one warm-up step bounds the CPU time; later warm-ups repeat the same work
    t0 = time.perf_counter()
    steps = 0
    budget = 120.0
    while steps < args.steps and time.perf_counter() - t0 < budget:
        rc, st = o.advance(nsteps=1)
        steps += 1
    dt = time.perf_counter() - t0
    val = prob.ncalc * steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "cell-timesteps/s", "n_gpus": ws,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / max(steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args, prob),
            "cpu_baseline": {"value": val, "unit": "cell-timesteps/s", "cores": threads, "kind": "port",
                             "sample": f"{steps} step(s) of the workload (bounded to {budget:.0f} s)"},
            "e2e": {"value": val, "unit": "cell-timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


METRIC = "cell-timesteps/s"


def workload_config(args, prob):
    prm = prob.params
    prec = {0: "ILU(0)/DILU", 1: "AMG"}[prm["precon_type"]]
    return {"workload": f"{prob.name} {prob.nx}x{prob.ny}x{prob.nz} ({prob.ncalc} cells)",
            "solver": f"Newton + BiCGStab + {prec}" + (" (reference quirks)" if prm["ref_quirks"] else ""),
            "precision": "fp64" if prm["precision"] == 0 else "mixed (fp32 V-cycle, bf16 coarse)",
            "newton_tol": f"{prm['criteria']} x max|h| (relative)" if prm["criteria_rel"] else prm["criteria"],
            "l2": "inputs larger than L2 (126 MB)" if prob.ncalc * 8 * 20 > 126e6 else "small case, L2 resident",
            "parallelism": f"replicas x{args.gpus}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hetero", choices=["hetero", "box", "large"])
    ap.add_argument("--shape", default="")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--precon", default="", choices=["", "ilu", "amg"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    rank, ws, dist = dist_setup()
    from msg123_b200 import build
    if rank == 0 and build.needs_build():
        build.build()
    barrier(dist)
    from msg123_b200.solver import GpuSolver, launch_count
    prob = make_problem(args, rank)
    g = GpuSolver(prob)
    g.init_state()
    # warm-up steps (untimed)
    rc, st_w = g.advance(nsteps=args.warmup)
    barrier(dist)
    l0 = launch_count()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        rc, st = g.advance(nsteps=args.steps)
    launches = launch_count() - l0
    ms = g.timers()["total_ms"]
    tmax = allmax(dist, ms)
    cells_steps = allsum(dist, float(prob.ncalc * st["accepted"]))
    value = cells_steps / (tmax * 1e-3)

    # kernel timings for the roofline (same context, state of the last timed step)
    peaks, src = load_peaks()
    hbm = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    kt = {}
    for which in (0, 1, 2):
        t = g.kernel_time(which, reps=10)
        kt[which] = t
    dom = 2   # the assembly pass is timed as the dominant bandwidth kernel
    achieved = ALG_BYTES[dom] * prob.ncalc / (kt[dom] * 1e-3) / 1e9
    spmv_gbs = ALG_BYTES[0] * prob.ncalc / (kt[0] * 1e-3) / 1e9

    # end-to-end through the public API with host-resident state
    e2e = None
    if not args.no_e2e:
        s = g.get_state()
        h_new, h_old, s_old, surf = s["head_new"], s["head_old"], s["srat_old"], s["surf_head"]
        N, S = prob.ncalc, prob.ncals
        barrier(dist)
        t0 = time.perf_counter()
        acc = 0
        for _ in range(args.steps):
            g.set_state(head_new=h_new, head_old=h_old, srat_old=s_old, surf_head=surf)
            rc2, st2 = g.advance(nsteps=1)
            s2 = g.get_state()
            h_old, s_old, surf = s2["head_new"], s2["srat_new"], s2["surf_head"]
            h_new = h_old
            acc += st2["accepted"]
        te = time.perf_counter() - t0
        te = allmax(dist, te)
        e2e = {"value": allsum(dist, float(prob.ncalc * acc)) / te, "unit": "cell-timesteps/s",
               "h2d_bytes_per_step": 3 * N * 8 + S * 8, "d2h_bytes_per_step": 5 * N * 8 + S * 8,
               "note": "state copied in and out through msg_gpu_set_state / msg_gpu_get_state every step"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, make_problem(args, 0))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-timesteps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tmax / max(st["accepted"], 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prob.params["precision"] == 0 else "f64+f32",
            "data": "synthetic", "config": workload_config(args, prob),
            "newton": {"accepted": st["accepted"], "rejected": st["rejected"], "newton_total": st["newton_total"],
                       "krylov_total": st["krylov_total"], "backtracks": st["back_total"],
                       "simulated_s": st["current_t"]},
            "roofline": {"kernel": KERNEL_NAMES[dom], "bound": "hbm", "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "peak_source": src,
                         "alg_bytes_per_cell": ALG_BYTES[dom], "ms_per_launch": kt[dom], "traffic": None,
                         "spmv_gbs": spmv_gbs, "spmv_frac": spmv_gbs / hbm,
                         "kernel_ms": {KERNEL_NAMES[k]: v for k, v in kt.items()}},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
        }
        print(json.dumps(line))
    g.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
