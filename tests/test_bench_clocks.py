"""bench.py's clock sampler on the host, against a stand-in `nvidia-smi` that
prints timestamped CSV samples: only samples taken inside the timed region
count, throttle flags are read, and a region shorter than one sampling
interval still reports the nearest sample."""
import os
import stat
import time

import pytest

FAKE = r"""#!/bin/sh
# stand-in for nvidia-smi --query-gpu=... -lms 50: idle clock first, then busy
i=0
while true; do
  ts=$(date +"%Y/%m/%d %H:%M:%S.%3N")
  if [ -f "$MARK" ]; then clk=1965; else clk=120; fi
  echo "$ts, 0, $clk, 1965, 500.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active"
  i=$((i+1))
  sleep 0.05
done
"""


@pytest.fixture
def fake_smi(tmp_path, monkeypatch):
    exe = tmp_path / "nvidia-smi"
    exe.write_text(FAKE)
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR | stat.S_IXGRP | stat.S_IXOTH)
    mark = tmp_path / "busy"
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    monkeypatch.setenv("MARK", str(mark))
    return mark


def test_clock_sampler_keeps_the_timed_region(fake_smi):
    import bench
    s = bench.ClockSampler(0)
    fake_smi.write_text("busy")  # the GPU is busy from here on
    s.start()
    time.sleep(0.4)
    c = s.stop()
    assert c is not None and c["in_window"]
    assert c["samples"] >= 4
    assert c["sm_mhz"] == 1965.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"]


def test_clock_sampler_short_region_reports_nearest_sample(fake_smi):
    import bench
    fake_smi.write_text("busy")
    s = bench.ClockSampler(0)
    s.start()
    c = s.stop()  # a region shorter than one interval
    assert c is not None and c["samples"] == 1
    assert c["sm_mhz"] == 1965.0
