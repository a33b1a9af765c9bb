"""Host-side pieces of bench.py that decide what its JSON line reports, on
the CPU: the clock sampler keeps only the nvidia-smi samples taken inside
the timed region (the throttle reasons and the median SM clock the line
carries are the timed region's, not the warm-up's), and the per-kernel
algorithmic byte counts follow the compact dealiased layout."""

import datetime
import importlib.util
import os
import tempfile

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("hit3d_bench", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _Done:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        pass


def _sampler(bench, rows):
    cs = bench.ClockSampler.__new__(bench.ClockSampler)
    cs.p = _Done()
    cs.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    cs.f.write("".join(rows))
    cs.f.flush()
    return cs


def _row(t, mhz, power_cap):
    act = "Active" if power_cap else "Not Active"
    return (f"{t.strftime('%Y/%m/%d %H:%M:%S.%f')[:-3]}, 0, {mhz}, 1965, 700.00, 0x0, Not Active, "
            f"Not Active, Not Active, {act}\n")


def test_clock_samples_are_those_of_the_timed_region(bench):
    t = datetime.datetime(2026, 1, 2, 3, 4, 5)
    ms = datetime.timedelta(milliseconds=1)
    # samples every 200 ms; the power cap is active only during the warm-up
    rows = [_row(t + 200 * i * ms, 1500 + i, i < 3) for i in range(12)]
    got = _sampler(bench, rows).stop(t + 1000 * ms, t + 1600 * ms)
    # window widened by one sample period: 800 .. 1800 ms
    assert got["samples"] == 6
    assert got["reasons"] == []
    assert got["sm_mhz"] == 1506.5
    assert got["sm_max_mhz"] == 1965.0
    # without a window every sample counts, the warm-up's throttle reason too
    allrows = _sampler(bench, rows).stop()
    assert allrows["samples"] == 12 and allrows["reasons"] == ["sw_power_cap"]


def test_clock_window_without_samples_falls_back_to_all(bench):
    t = datetime.datetime(2026, 1, 2, 3, 4, 5)
    rows = [_row(t + datetime.timedelta(seconds=i), 1965, False) for i in range(3)]
    later = t + datetime.timedelta(hours=1)
    assert _sampler(bench, rows).stop(later, later)["samples"] == 3


def test_kernel_bytes_follow_the_compact_layout(bench):
    # 512^3 dealiased, padding excluded: compact spectral A = 341 x 341 x 171,
    # x-physical Bx = 512 x 341 x 171, x,y-physical Cx = 512 x 512 x 171
    # (complex64)
    b = bench.kernel_alg_bytes(512)
    A, Bx, Cx = 341 * 341 * 171, 512 * 341 * 171, 512 * 512 * 171
    assert b["y-inverse"] == (6 * Bx + 6 * Cx) * 8
    assert b["z-pass"] == (6 * Cx + 3 * Cx) * 8
    assert b["y-forward"] == (3 * Cx + 3 * Bx) * 8
    assert b["x-inverse"] == (3 * A + 6 * Bx) * 8
    assert bench.spectral_bytes(512) == 538968064
