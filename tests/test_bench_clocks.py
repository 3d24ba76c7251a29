"""The clock sampler of bench.py (CPU): samples taken while the timed region
runs, the pre-region sample left out, throttle reasons collected, and the
line it reports without nvidia-smi.  A stand-in nvidia-smi prints rows in
the --query-gpu order that bench.py asks for."""
import importlib.util
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

FAKE = """#!{py}
import sys, time
ms = int(sys.argv[sys.argv.index("-lms") + 1])
time.sleep(0.1)
i = 0
while True:
    cap = "Active" if i == {cap_at} else "Not Active"
    print(f"0, {{1900 + i}}, 1965, 700.0, 0x4, Not Active, Not Active, Not Active, {{cap}}", flush=True)
    i += 1
    time.sleep(ms / 1000)
"""


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _fake_smi(tmp_path, monkeypatch, cap_at):
    d = tmp_path / "bin"
    d.mkdir()
    p = d / "nvidia-smi"
    p.write_text(FAKE.format(py=sys.executable, cap_at=cap_at))
    p.chmod(0o755)
    monkeypatch.setenv("PATH", f"{d}{os.pathsep}{os.environ.get('PATH', '')}")


def test_samples_cover_the_region(tmp_path, monkeypatch):
    _fake_smi(tmp_path, monkeypatch, cap_at=3)
    clk = _bench().Clocks(0)
    clk.start()
    assert clk.first >= 1  # the sampler was running before the region began
    time.sleep(0.4)
    out = clk.stop()
    assert out["samples"] >= 4
    assert out["sm_max_mhz"] == 1965.0
    # the pre-region sample (1900 MHz) is left out of the median
    assert out["sm_mhz"] > 1900.0
    assert out["reasons"] == ["sw_power_cap"]


def test_short_region_keeps_the_last_sample(tmp_path, monkeypatch):
    _fake_smi(tmp_path, monkeypatch, cap_at=-1)
    clk = _bench().Clocks(0)
    clk.start()
    out = clk.stop()  # ends before the next sample
    assert out["samples"] >= 1
    assert out["reasons"] == []


def test_without_nvidia_smi(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    clk = _bench().Clocks(0)
    clk.start()
    assert clk.stop() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
