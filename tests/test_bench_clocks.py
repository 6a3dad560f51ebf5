"""bench.py's clock sampler keeps the nvidia-smi samples taken inside the
timed region and reads the throttle reasons from them (a stand-in
nvidia-smi on PATH prints timestamped samples; no GPU)."""
import os
import stat
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

FAKE = """#!{py}
import datetime, sys, time
while True:
    now = datetime.datetime.now().strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    print(f"{{now}}, 0, 1800, 1965, 950.0, 0x4, Not Active, Not Active, Not Active, Active",
          flush=True)
    time.sleep(0.1)
"""


def test_samples_inside_the_region(tmp_path, monkeypatch):
    import bench
    fake = tmp_path / "nvidia-smi"
    fake.write_text(FAKE.format(py=sys.executable))
    fake.chmod(fake.stat().st_mode | stat.S_IEXEC)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    s = bench.ClockSampler(0)
    s.start()
    time.sleep(0.45)
    out = s.stop()
    assert out["samples_in_region"] >= 2
    assert out["samples"] == out["samples_in_region"]
    assert out["sm_mhz"] == 1800.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]


def test_without_nvidia_smi(tmp_path, monkeypatch):
    import bench
    monkeypatch.setenv("PATH", str(tmp_path))
    s = bench.ClockSampler(0)
    s.start()
    out = s.stop()
    assert out["sm_mhz"] is None and out["reasons"] == ["nvidia-smi unavailable"]
