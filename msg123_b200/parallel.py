"""Multi-GPU ensemble: members sharded over ranks, one process per GPU.

Ensemble members are independent realisations, so they shard with no data-path
collective.  Every rank computes the same assignment -- a greedy longest-processing-time
bin-pack on cells x expected Newton iterations per step (the expected count grows with
the member's lnKs spread) -- builds only its own members on its GPU and advances them with
the batched driver (msg_gpu_ensemble_advance).  Per-member statistics are gathered on the
host at the end; throughput = all members' cells x accepted steps / the slowest rank's time.
A rank whose members fail still joins that gather, carrying the error, so every rank stops
with the same message instead of waiting in the collective for a rank that left.

The reference runs one realisation per (MPI) job; this replaces launching many jobs.
"""
import time

from .config import member_draw


def expected_newton(sigma):
    """Newton iterations per step expected for a member with lnKs spread `sigma`
    (heterogeneity lengthens the Newton paths; only the ordering matters for the packing)."""
    return 4.0 + 4.0 * float(sigma)


def member_work(seeds):
    """Work estimate per member: cells x expected Newton iterations."""
    out = []
    for s in seeds:
        (nx, ny, nz), sigma = member_draw(s)
        out.append(nx * ny * nz * expected_newton(sigma))
    return out


def assign(work, world_size):
    """Greedy LPT bin-pack: members by decreasing work, each to the least-loaded rank
    (ties to the lower rank).  Returns (members per rank, load per rank); deterministic, so
    every rank computes the same answer without communicating."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(work)), key=lambda k: (-work[k], k))
    parts = [[] for _ in range(world_size)]
    load = [0.0] * world_size
    for k in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += work[k]
    for p in parts:
        p.sort()
    return parts, load


def gpu_runner(seeds, nsteps, autotune=True):
    """Build this rank's members on the current GPU, advance them `nsteps` accepted steps
    each, return (per-member stats in `seeds` order, seconds)."""
    from .ensemble import Ensemble
    ens = Ensemble(seeds=seeds)
    try:
        ens.init_state()
        if autotune:
            ens.autotune(probe_steps=1)
        dt, stats = ens.advance(nsteps)
        for s, c in zip(stats, ens.cells):
            s["cells"] = int(c)
        return stats, dt
    finally:
        ens.close()


def run(nmembers, nsteps, rank=0, world_size=1, dist=None, runner=gpu_runner, seed0=0):
    """Run the sharded ensemble.  Returns, on every rank, a dict with the assignment, the
    per-member statistics (member order) and the aggregate throughput."""
    seeds = [seed0 + k for k in range(nmembers)]
    parts, load = assign(member_work(seeds), world_size)
    mine = [seeds[k] for k in parts[rank]]
    t0 = time.perf_counter()
    err = None
    try:
        stats, dt = runner(mine, nsteps) if mine else ([], 0.0)
    except Exception as e:   # reported to every rank by the gather below, which all ranks reach
        stats, dt, err = [], 0.0, f"{type(e).__name__}: {e}"
    wall = time.perf_counter() - t0
    local = {"rank": rank, "members": parts[rank], "stats": stats, "seconds": dt, "wall": wall, "error": err}
    if dist is not None and world_size > 1:
        gathered = [None] * world_size
        dist.all_gather_object(gathered, local)
    else:
        gathered = [local]
    failed = [(g["rank"], g["error"]) for g in gathered if g["error"]]
    if failed:
        raise RuntimeError("ensemble failed on " + "; ".join(f"rank {r}: {m}" for r, m in failed))
    per_member = [None] * nmembers
    for g in gathered:
        for k, s in zip(g["members"], g["stats"]):
            per_member[k] = s
    tmax = max(g["seconds"] for g in gathered)
    cell_steps = float(sum(s["cells"] * s["accepted"] for s in per_member if s is not None))
    return {"parts": parts, "load": load, "stats": per_member, "seconds_max": tmax,
            "throughput": cell_steps / tmax if tmax > 0 else 0.0}
