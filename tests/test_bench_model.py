"""bench.py without a GPU: the algorithmic-byte model behind the V-cycle roofline entry
(counted by hand on small hierarchies), the clocks summary, the measured-peaks reader, and
dry runs of the whole benchmark -- one rank, and two ranks over gloo -- with stand-ins for
the CUDA solver, so every key of the JSON line and the multi-rank reductions are checked."""
import importlib.util
import os

import pytest

_spec = importlib.util.spec_from_file_location("bench", os.path.join(os.path.dirname(__file__), "..", "bench.py"))
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)


def test_two_levels_dense_coarsest():
    # fine 1000 cells, coarse 100 rows solved by the dense inverse, P with 1500 entries
    sizes = [(1000, 5800, 0), (100, 900, 1500)]
    fine = 20 * 1000 + 40 * 1000 + 2 * 40 * 1000 + 4 * 1000            # first, 1 pre, 2 post, FP64 out
    res = 40 * 1000
    restrict = 4 * 100 + 8 * 1500 + 4 * 1000 + 4 * 100
    prolong = 4 * 1000 + 8 * 1500 + 4 * 100 + 8 * 1000
    dense = 8 * 100 * 100 + 8 * 100
    assert bench.vcycle_bytes(sizes, 2, 128) == pytest.approx(fine + res + restrict + prolong + dense)


def test_three_levels_smoothed_coarsest():
    # coarsest too large for the dense inverse: it is smoothed like the middle level
    sizes = [(1000, 5800, 0), (200, 2000, 1500), (150, 1500, 400)]
    coarse_max = 100
    fine = 20 * 1000 + 40 * 1000 + 2 * 40 * 1000 + 4 * 1000
    t01 = 40 * 1000 + (4 * 200 + 8 * 1500 + 4 * 1000 + 4 * 200) + (4 * 1000 + 8 * 1500 + 4 * 200 + 8 * 1000)
    sw1 = 20 * 200 + 6 * 2000
    mid = 12 * 200 + 3 * sw1
    t12 = sw1 + (4 * 150 + 8 * 400 + 4 * 200 + 4 * 150) + (4 * 200 + 8 * 400 + 4 * 150 + 8 * 200)
    sw2 = 20 * 150 + 6 * 1500
    last = 12 * 150 + 3 * sw2
    assert bench.vcycle_bytes(sizes, 2, coarse_max) == pytest.approx(fine + t01 + mid + t12 + last)


def test_no_sweeps():
    sizes = [(1000, 5800, 0), (100, 900, 1500)]
    got = bench.vcycle_bytes(sizes, 0, 128)
    fine = 16 * 1000 + 12 * 1000
    res = 40 * 1000
    restrict = 4 * 100 + 8 * 1500 + 4 * 1000 + 4 * 100
    prolong = 4 * 1000 + 8 * 1500 + 4 * 100 + 8 * 1000
    assert got == pytest.approx(fine + res + restrict + prolong + 8 * 100 * 100 + 8 * 100)


def test_clock_summary_from_samples():
    """The clocks key of the bench line: median SM clock, highest max clock and every
    throttle reason seen Active in any sample (nvidia-smi csv, noheader, nounits)."""
    cs = bench.ClockSampler()
    assert cs.summary()["reasons"] == ["unsampled"]
    cs.samples = [["1965", "1965", "700.1", "Not Active", "Not Active", "Not Active", "Not Active"],
                  ["1950", "1965", "980.0", "Not Active", "Not Active", "Not Active", "Active"],
                  ["1980", "1965", "990.5", "Not Active", "Not Active", "Not Active", "Active"],
                  ["[N/A]", "1965", "[N/A]", "Not Active", "Active", "Not Active", "Not Active"]]
    s = cs.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 4
    assert s["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


def test_load_peaks(tmp_path):
    import json
    assert bench.load_peaks(str(tmp_path / "absent.json"))[2] == "fallback"
    p = tmp_path / "peaks.json"
    p.write_text(json.dumps({"hbm_gbs": 6543.7, "bf16_tflops": 1642.7, "bf16_tflops_sustained": 1400.0}))
    assert bench.load_peaks(str(p)) == (6543.7, 1642.7, "measured")
    p.write_text(json.dumps({"hbm_gbs": {"value": 6500.0}, "bf16_tflops": {"value": 1600.0}}))
    assert bench.load_peaks(str(p)) == (6500.0, 1600.0, "measured")
    p.write_text("{not json")
    hbm, tc, src = bench.load_peaks(str(p))
    assert (hbm, tc) == (6650.0, 1590.0) and src.startswith("fallback")


class _FakeSolver:
    """Stands in for GpuSolver in a dry run of bench.main: fixed kernel times, one AMG level
    pair, a state of the right size, a clock that stops at the context's end time."""

    def __init__(self, prob, **kw):
        self.prob, self.params = prob, dict(prob.params, **kw)
        self.t = 0.0

    def init_state(self):
        pass

    def copy_state_from(self, other):
        self.t = other.t

    def advance(self, nsteps=1, **kw):
        n = 0
        while n < nsteps and self.t < self.params["end_time"]:
            self.t = min(self.t + 600.0, self.params["end_time"])
            n += 1
        self.last_n = n
        return 0, dict(accepted=n, rejected=0, newton_total=5 * n, krylov_total=5 * n,
                       back_total=0, current_t=self.t, delt=600.0, status=0)

    def timers(self):
        """5 ms of device time per step of the last advance call."""
        n = getattr(self, "last_n", 0)
        return {"assembly_ms": 1.5 * n, "krylov_ms": 2.0 * n, "amg_setup_ms": 0.5 * n, "residual_ms": 1.0 * n,
                "total_ms": 5.0 * n}

    def kernel_time(self, which, reps=1):
        return {0: 0.01, 1: 0.02, 2: 0.03, 3: 0.05, 4: 1.0, 5: 0.2}[which]

    def amg_sizes(self):
        n = self.prob.ncalc
        return [(n, 6 * n, 0), (n // 8, n, n)]

    def get_state(self, out=None):
        import numpy as np
        out = out if out is not None else {}
        for k, a in out.items():
            a[:] = np.asarray(self.prob.head0 if k.startswith("head") else 0.5)[:a.size] if k.startswith("head") \
                else 0.5
        return out

    def set_state(self, **kw):
        pass

    def srat_rperm(self, head):
        import numpy as np
        return np.full(head.size, 0.5), np.ones(head.size), np.zeros(head.size)

    def guess_fallbacks(self):
        return 0

    def guess_rejected(self):
        return 0

    def close(self):
        pass


@pytest.mark.parametrize("extra", [["--no-cpu", "--no-arms", "--no-e2e"],
                                   ["--cpu-shape", "8x8x4", "--no-e2e"],
                                   ["--no-cpu", "--no-arms"],
                                   ["--no-cpu"]])
def test_bench_main_dry_run(monkeypatch, capsys, extra):
    """bench.main on the CPU with stand-ins for the CUDA solver and the network: the JSON
    line carries every key of the contract, with values derived from the stand-ins."""
    import json
    import sys
    from msg123_b200 import learned, solver, train_guess
    monkeypatch.setattr(solver, "GpuSolver", _FakeSolver)
    monkeypatch.setattr(solver, "launch_count", lambda: 0)
    monkeypatch.setattr(learned, "Cnn", lambda seed=0: type("C", (), {"attach": lambda s, g: None,
                                                                       "close": lambda s: None})())
    monkeypatch.setattr(train_guess, "load", lambda c: c)
    import torch
    empty = torch.empty
    monkeypatch.setattr(torch, "empty", lambda *a, pin_memory=False, **k: empty(*a, **k))   # no CUDA here
    monkeypatch.setattr(sys, "argv", ["bench.py", "--workload", "hetero", "--shape", "8x8x4", "--steps", "2",
                                      "--warmup", "3"] + extra)
    bench.main()
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "roofline", "cpu_baseline", "e2e",
              "gpu_launches", "clocks"):
        assert k in line, k
    assert line["value"] == pytest.approx(256 * 2 / 10e-3)
    r = line["roofline"]
    # the assembly pair (make_matvec, kernel_time 2) is the line's dominant kernel; the others sit beside it
    assert r["ms_per_launch"] == 0.03 and r["unit"] == "GB/s" and 0 < r["frac"]
    assert r["alg_bytes_per_cell"] == 280.0 and r["traffic"] == pytest.approx((93.8 + 170.8) * 256)
    assert r["others"]["calc_func (vG pass + flux pass)"]["ms"] == 0.02
    assert r["others"]["mixed V-cycle, all levels"]["ms"] == 0.05
    assert r["vcycle_mixed_ms"] == 0.05 and line["config"]["workload"].startswith("hetero 8x8x4")
    assert line["newton"]["accepted"] == 2 and line["newton"]["simulated_s"] == 3000.0 and line["window_start_s"] == 1800.0
    if "--no-arms" not in extra:                      # every arm stops at the value path's end time
        for name in ("mixed_extrapolation", "fp64_extrapolation", "plain_fp64", "value"):
            assert line["arms"][name]["simulated_s"] == 3000.0
        assert line["speedup_over_plain_fp64"] == pytest.approx(1.0)
    if "--no-arms" not in extra and "--no-e2e" not in extra:   # FP64 on the value path's own steps
        assert line["errors_vs_fp64"]["head_rel"] == 0.0 and line["errors_vs_fp64"]["steps"] == 2
    if "--no-e2e" not in extra:                       # pinned host state in and out every step
        e = line["e2e"]
        assert e["h2d_bytes_per_step"] == 3 * 256 * 8 + 64 * 8 and e["d2h_bytes_per_step"] == 2 * 256 * 8 + 64 * 8
        assert e["value"] > 0 and e["accepted"] == 2 and e["same_window_as_value"]
    if "--no-cpu" not in extra:                       # the oracle really ran on the 8x8x4 sample
        cb = line["cpu_baseline"]
        assert cb["kind"] == "port" and cb["value"] > 0 and "8x8x4" in cb["sample"]
        assert cb["nproc"] >= 1 and "cpu_model" in cb
        assert line["reference_method_gpu"]["steps"] >= 1


def _bench_rank(rank, world, port, q):
    """One rank of a two-rank bench run over gloo, with the stand-ins of the dry run."""
    import contextlib
    import io
    import sys
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), LOCAL_RANK=str(rank),
                      WORLD_SIZE=str(world))
    from msg123_b200 import learned, solver, train_guess
    solver.GpuSolver = _FakeSolver
    solver.launch_count = lambda: 0
    learned.Cnn = lambda seed=0: type("C", (), {"attach": lambda s, g: None, "close": lambda s: None})()
    train_guess.load = lambda c: c
    sys.argv = ["bench.py", "--workload", "hetero", "--shape", "8x8x4", "--steps", "2", "--warmup", "3",
                "--gpus", str(world), "--no-cpu", "--no-arms", "--no-e2e"]
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        bench.main()
    q.put((rank, out.getvalue()))


def test_bench_two_ranks_over_gloo():
    """bench.py under two ranks (gloo on CPU): only rank 0 prints, and the value is the
    cells x steps of both ranks over the slowest rank's time."""
    import json
    import socket
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_bench_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outs = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert outs[1].strip() == ""
    line = json.loads(outs[0].strip().splitlines()[-1])
    assert line["n_gpus"] == 2 and line["value"] == pytest.approx(2 * 256 * 2 / 10e-3)
    assert line["config"]["parallelism"] == "replicas x2"
