"""The autotuner's choices on a stand-in integrator with scripted kernel
times (no GPU): per-class picks, the whole-step comparison of the deferred
last RK stage (variant 3 moves time from the RK class to the x sweep) and of
the fused y and z sweeps (y variant 3: one pass in place of two), the
refusal of RK variants under a source term, and the cache."""
import pytest

from miso_b200 import _lib, autotune


class FakeInteg:
    """Kernel times per class as functions of the variants set."""

    def __init__(self, defer_gain, refuse_rk=(), fused_ms=20.0):
        self.var = {0: 3, 1: 0, 2: 3, 3: 0}
        self.chunks = (64, 128)
        self.defer_gain = defer_gain
        self.fused_ms = fused_ms
        self.refuse_rk = refuse_rk
        self.config, self.precision = {}, "fp32_split"

    def get_variant(self, kc):
        return self.var[kc]

    def set_variant(self, kc, v):
        if kc == 0 and v in self.refuse_rk:
            raise _lib.MisoError(_lib.ERR_STATE, "refused")
        self.var[kc] = v

    def set_chunks(self, rk, av):
        self.chunks = (rk, av)

    def set_timing(self, on):
        pass

    def run(self, n, graph=False):
        pass

    def sync(self):
        pass

    def timing_report(self):
        rk = {0: 4.0, 1: 5.0, 2: 3.3, 3: 3.3 - self.defer_gain}[self.var[0]]
        # variant 3 takes the update into the x sweep: the sweep pays part of it
        avx = {0: 4.3, 1: 6.0, 2: 5.2}[self.var[1]] + (0.5 * 4 * self.defer_gain
                                                        if self.var[0] == 3 else 0.0)
        chunk = 0.01 * abs(self.chunks[0] - 64) / 64
        rep = {"rk_stage": {"ms": 4 * (rk + chunk), "launches": 4},
               "av_x": {"ms": avx, "launches": 1}}
        if self.var[2] == 3:  # the fused y and z sweeps: one pass
            rep["av_yz"] = {"ms": self.fused_ms, "launches": 1}
        else:
            rep["av_y"] = {"ms": {0: 4.3, 1: 6.0, 2: 5.2}[self.var[2]], "launches": 1}
            rep["av_z"] = {"ms": {0: 5.0, 1: 7.0, 2: 6.2}[self.var[3]], "launches": 1}
        return rep


@pytest.fixture
def cache(tmp_path, monkeypatch):
    monkeypatch.setenv("MISO_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(autotune, "_key", lambda integ: "fake:key")


def test_deferred_stage_kept_when_the_whole_step_gains(cache):
    integ = FakeInteg(defer_gain=0.8)  # RK -3.2 ms over 4 stages, x sweep +1.6 ms
    choice = autotune.autotune(integ, steps=1)
    assert choice["rk_stage"] == 3 and integ.get_variant(0) == 3
    assert (choice["av_x"], choice["av_y"], choice["av_z"]) == (0, 0, 0)
    assert choice["rk_chunk"] == 64
    again = autotune.autotune(integ)
    assert again.get("cached") and again["rk_stage"] == 3


def test_deferred_stage_dropped_when_the_step_loses(cache):
    integ = FakeInteg(defer_gain=-0.2)  # variant 3 slower in both classes
    choice = autotune.autotune(integ, steps=1)
    assert choice["rk_stage"] == 2 and integ.get_variant(0) == 2


def test_refused_variants_are_skipped(cache):
    integ = FakeInteg(defer_gain=0.8, refuse_rk=(0, 1))  # a source term pins RK to 2 / 3
    choice = autotune.autotune(integ, steps=1)
    assert choice["rk_stage"] in (2, 3)


def test_fused_sweeps_kept_when_the_step_gains(cache):
    integ = FakeInteg(defer_gain=0.8, fused_ms=7.0)  # 7.0 ms against 4.3 + 5.0
    choice = autotune.autotune(integ, steps=1)
    assert choice["av_y"] == 3 and integ.get_variant(2) == 3
    assert choice["ms"]["av_y"] == 7.0 and "av_z" not in choice["ms"]


def test_fused_sweeps_dropped_when_the_step_loses(cache):
    integ = FakeInteg(defer_gain=0.8, fused_ms=9.5)
    choice = autotune.autotune(integ, steps=1)
    assert choice["av_y"] == 0 and integ.get_variant(2) == 0
