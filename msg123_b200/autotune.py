"""Launch-shape autotuner.

Times the candidate block sizes of the kernels whose launch shape is free (the van
Genuchten/storage pass and the level-1 V-cycle smoother; kernels with reductions keep a
fixed shape so results never depend on the tuning) with msg_gpu_kernel_time on the
solver's own state, and caches the choice per (nx, ny, nz, precision, kr form) in a JSON
file ($MSG123_TUNE_CACHE, default ~/.cache/msg123_b200/tuning.json).
"""
import json
import os

CELL_BLOCKS = (128, 256, 512)
SMOOTH_BLOCKS = (128, 256, 512, 1024)


def cache_path():
    return os.environ.get("MSG123_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "msg123_b200", "tuning.json"))


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _save(d):
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def key(solver):
    p = solver.prob
    return f"{p.nx}x{p.ny}x{p.nz}:p{solver.params['precision']}:v{solver.params.get('vg_form', 0)}"


def tune(solver, reps=5, use_cache=True):
    """Pick (blk_cell, blk_smooth) for this solver's grid; apply and return them.
    The solver must have assembled a system (one advance) so the V-cycle exists."""
    d = _load() if use_cache else {}
    k = key(solver)
    if k in d:
        bc, bs = d[k]["blk_cell"], d[k]["blk_smooth"]
        solver.set_tuning(bc, bs)
        return bc, bs, d[k]
    times_c = {}
    for bc in CELL_BLOCKS:
        solver.set_tuning(bc, 256)
        times_c[bc] = solver.kernel_time(2, reps=reps)
    bc = min(times_c, key=times_c.get)
    times_s = {}
    for bs in SMOOTH_BLOCKS:
        solver.set_tuning(bc, bs)
        times_s[bs] = solver.kernel_time(3, reps=reps)
    bs = min(times_s, key=times_s.get)
    solver.set_tuning(bc, bs)
    rec = {"blk_cell": bc, "blk_smooth": bs, "make_matvec_ms": times_c, "precond_ms": times_s}
    d = _load()
    d[k] = rec
    try:
        _save(d)
    except OSError:
        pass
    return bc, bs, rec
