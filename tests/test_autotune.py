"""The launch-shape autotuner's selection and cache logic, with a stand-in solver whose
kernel times depend on the block sizes (no GPU)."""
from types import SimpleNamespace

from msg123_b200 import autotune


class FakeSolver:
    def __init__(self, shape=(64, 48, 32), precision=1, vg_form=1, best=(256, 512)):
        self.prob = SimpleNamespace(nx=shape[0], ny=shape[1], nz=shape[2])
        self.params = dict(precision=precision, vg_form=vg_form)
        self.best, self.tuning, self.calls = best, None, 0

    def set_tuning(self, bc, bs):
        self.tuning = (bc, bs)

    def kernel_time(self, which, reps=5):
        self.calls += 1
        bc, bs = self.tuning
        return 1.0 + abs(bc - self.best[0]) / 1000.0 if which == 2 else 2.0 + abs(bs - self.best[1]) / 1000.0


def test_tune_picks_fastest_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("MSG123_TUNE_CACHE", str(tmp_path / "tune.json"))
    s = FakeSolver()
    bc, bs, rec = autotune.tune(s)
    assert (bc, bs) == (256, 512) and s.tuning == (256, 512)
    assert s.calls == len(autotune.CELL_BLOCKS) + len(autotune.SMOOTH_BLOCKS)
    s2 = FakeSolver(best=(128, 128))                 # same key: served from the cache, no timing
    assert autotune.tune(s2)[:2] == (256, 512) and s2.calls == 0 and s2.tuning == (256, 512)
    s3 = FakeSolver(vg_form=0, best=(512, 1024))     # another kr form is another key
    assert autotune.tune(s3)[:2] == (512, 1024) and s3.calls > 0
    s4 = FakeSolver(best=(128, 128))
    assert autotune.tune(s4, use_cache=False)[:2] == (128, 128)


def test_unwritable_cache_is_not_fatal(tmp_path, monkeypatch):
    blocker = tmp_path / "file"
    blocker.write_text("x")
    monkeypatch.setenv("MSG123_TUNE_CACHE", str(blocker / "sub" / "tune.json"))
    assert autotune.tune(FakeSolver())[:2] == (256, 512)
