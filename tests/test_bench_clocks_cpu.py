"""bench.py's clock sampler against a stand-in nvidia-smi on PATH: it waits
for the first sample before returning from start(), reports the median SM
clock, the maximum and every throttle reason that was active, and reports
"unavailable" when nvidia-smi cannot be started."""
import importlib.util
import os
import pathlib
import stat

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


FAKE = """#!/bin/sh
sleep 0.2
echo "0, 1965, 1965, 612.3, 0x0, Not Active, Not Active, Not Active, Not Active"
echo "0, 1900, 1965, 998.0, 0x4, Not Active, Not Active, Not Active, Active"
echo "0, 1950, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active"
echo "garbage line"
sleep 30
"""


@pytest.fixture
def fake_smi(tmp_path, monkeypatch):
    p = tmp_path / "nvidia-smi"
    p.write_text(FAKE)
    p.chmod(p.stat().st_mode | stat.S_IEXEC)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ.get('PATH', '')}")
    return p


def test_sampler_parses_clocks_and_reasons(fake_smi):
    bench = _bench()
    s = bench.ClockSampler(0)
    s.start()
    assert s.lines, "start() returns only after the first sample"
    ck = s.stop()
    assert ck["samples"] == 3
    assert ck["sm_mhz"] == 1950.0 and ck["sm_max_mhz"] == 1965.0
    assert ck["reasons"] == ["sw_power_cap"]


def test_sampler_without_nvidia_smi(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    bench = _bench()
    s = bench.ClockSampler(0)
    s.start()
    assert s.stop() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}

