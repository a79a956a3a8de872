"""The bench's clock sampler on the CPU, driven by a fake nvidia-smi: only rows stamped inside the timed region
count, and a region with no row inside it reports "unsampled" rather than a clock read before it."""

import sys
import textwrap
import time
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))

import bench  # noqa: E402

FAKE = textwrap.dedent("""
    import datetime, sys, time
    period, count, first_delay = float(sys.argv[1]), int(sys.argv[2]), float(sys.argv[3])
    def row(mhz):
        stamp = datetime.datetime.now().strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
        print(f"{stamp}, 0, {mhz}, 1965, 500.0, 0x0, Not Active, Not Active, Not Active, Not Active", flush=True)
    row(1000)                 # a row before the region starts
    time.sleep(first_delay)
    for n in range(count):
        row(1965)
        time.sleep(period)
    time.sleep(60)
""")


def fake_command(tmp_path, period, count, first_delay):
    script = tmp_path / "fake_smi.py"
    script.write_text(FAKE)
    return [sys.executable, str(script), str(period), str(count), str(first_delay)]


def test_rows_inside_the_region_are_the_only_ones_counted(tmp_path):
    sampler = bench.ClockSampler(None, command=fake_command(tmp_path, 0.05, 100, 0.1))
    with sampler:
        time.sleep(0.5)
    summary = sampler.summary()
    assert summary["sm_mhz"] == 1965.0  # the 1000 MHz row came before the region
    assert summary["samples"] >= 4
    assert summary["rows_outside_region"] >= 1
    assert summary["reasons"] == []


def test_a_region_without_rows_is_unsampled(tmp_path):
    sampler = bench.ClockSampler(None, command=fake_command(tmp_path, 0.05, 0, 0.0))
    with sampler:
        time.sleep(0.2)
    summary = sampler.summary()
    assert summary["sm_mhz"] is None
    assert summary["reasons"] == ["unsampled"]
    assert summary["samples"] == 0
