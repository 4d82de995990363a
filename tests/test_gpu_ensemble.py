"""Batched ensemble (uneven members advanced concurrently) and the autotuner.

Every member advanced through msg_gpu_ensemble_advance must give the same heads as
the same member advanced alone (the members share nothing but the GPU), and the
autotuned launch shapes must not change results."""
import numpy as np
import pytest

from msg123_b200.config import make_member

pytestmark = pytest.mark.gpu


def test_ensemble_members_match_solo_runs(tmp_path, monkeypatch):
    monkeypatch.setenv("MSG123_TUNE_CACHE", str(tmp_path / "tune.json"))
    from msg123_b200.ensemble import Ensemble, ENSEMBLE
    from msg123_b200.solver import GpuSolver
    ens = Ensemble(nmembers=6, seed0=40)
    ens.init_state()
    ens.advance(1, workers=3)
    info = ens.autotune(worker_candidates=(2, 6))
    rate, dt, stats, newton = ens.throughput(2)
    assert all(s["status"] == 0 and s["accepted"] == 2 for s in stats)
    assert len(set(newton)) >= 1
    for k in (0, 3, 5):
        p = make_member(40 + k)
        with GpuSolver(p, **ENSEMBLE) as g:
            g.init_state()
            g.advance(nsteps=1 + 1 + len((2, 6)) + 2)  # warm-up + autotune's probe step + two worker probes + timed
            h_solo = g.get_state()["head_new"]
        h_ens = ens.members[k].get_state()["head_new"]
        assert np.max(np.abs(h_ens - h_solo)) / np.max(np.abs(h_solo)) <= 1e-12, k
    print("ensemble", rate, info, newton)
    ens.close()


def test_ensemble_members_share_one_network():
    """One CNN attached to every member, members advanced by concurrent worker threads
    (guess_mode = 2): each member ends where it ends when advanced alone with that network."""
    from msg123_b200.ensemble import Ensemble, ENSEMBLE
    from msg123_b200.learned import Cnn
    from msg123_b200.solver import GpuSolver
    from msg123_b200.train_guess import load
    cnn = load(Cnn(seed=0))
    kw = dict(guess_mode=2, guess_select=0)
    ens = Ensemble(nmembers=4, seed0=60, **kw)
    for g in ens.members:
        cnn.attach(g)
    ens.init_state()
    dt, stats = ens.advance(4, workers=4)
    assert all(s["status"] == 0 and s["accepted"] == 4 for s in stats)
    for k in range(4):
        p = make_member(60 + k)
        o = dict(ENSEMBLE)
        o.update(kw)
        with GpuSolver(p, **o) as g:
            cnn.attach(g)
            g.init_state()
            g.advance(nsteps=4)
            h_solo = g.get_state()["head_new"]
        h_ens = ens.members[k].get_state()["head_new"]
        assert np.max(np.abs(h_ens - h_solo)) / np.max(np.abs(h_solo)) <= 1e-12, k
    ens.close()
    cnn.close()
