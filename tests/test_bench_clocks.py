"""The benchmark's clock summary (CPU): only samples taken inside the timed region count, throttle
reasons are read from the sampled flags, and a region shorter than the sampling period still gets
the samples nearest to it."""
import datetime
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _sampler(lines, t0, t1):
    sys.path.insert(0, str(ROOT))
    import bench
    c = bench.ClockSampler(0)
    fd, path = tempfile.mkstemp(suffix=".csv")
    with open(fd, "w") as f:
        f.write("\n".join(lines) + "\n")
    c.path, c.t0, c.t1 = path, t0, t1
    return c.summary()


def _row(ts, mhz, power=300.0, slow="Not Active", cap="Not Active"):
    stamp = datetime.datetime.fromtimestamp(ts).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    return f"{stamp}, 0, {mhz}, 1965, {power}, 0x0, {slow}, Not Active, Not Active, {cap}"


def test_only_samples_inside_the_region_count():
    t0 = 1_800_000_000.0
    lines = [_row(t0 - 1.0, 345), _row(t0 + 0.05, 1965), _row(t0 + 0.10, 1950, cap="Active"),
             _row(t0 + 0.15, 1965), _row(t0 + 2.0, 345, slow="Active")]
    s = _sampler(lines, t0, t0 + 0.2)
    assert s["samples"] == 3 and s["window"] == "timed region"
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]


def test_short_region_takes_the_nearest_samples():
    t0 = 1_800_000_000.0
    lines = [_row(t0 - 0.2, 1900), _row(t0 + 0.3, 1965), _row(t0 + 5.0, 345)]
    s = _sampler(lines, t0, t0 + 0.01)
    assert s["window"] == "nearest to the timed region" and s["samples"] == 2
    assert s["sm_mhz"] == (1900 + 1965) / 2


def test_no_samples_is_reported_as_unsampled():
    s = _sampler(["garbage"], 0.0, 1.0)
    assert s["reasons"] == ["unsampled"] and s["sm_mhz"] is None
