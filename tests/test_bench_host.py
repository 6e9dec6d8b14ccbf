"""Host-side pieces of bench.py that need no GPU: the clock sampler's
window filter and reason parsing, the angle-chunk schedule."""
import importlib.util
import pathlib

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _DoneProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def _line(sm, power_cap="Not Active", thermal="Not Active"):
    return f"0, {sm}, 1965, 700.0, 0x0, Not Active, Not Active, {thermal}, {power_cap}"


def test_clock_sampler_keeps_samples_inside_the_timed_window():
    b = _bench()
    c = b.ClockSampler(0)
    c.INTERVAL_MS = 0
    c.proc = _DoneProc()
    c.lines = [(9.0, _line(900, thermal="Active")), (10.1, _line(1965)), (10.6, _line(1950, power_cap="Active")),
               (11.2, _line(1000, thermal="Active"))]
    c.mark(10.0, 11.0)
    r = c.stop()
    assert r["samples"] == 2 and r["sm_max_mhz"] == 1965
    assert r["sm_mhz"] == np.median([1965, 1950])
    # the slowdowns outside the window are not reported
    assert r["reasons"] == ["sw_power_cap"]


def test_clock_sampler_short_window_keeps_nearest_samples():
    b = _bench()
    c = b.ClockSampler(0)
    c.INTERVAL_MS = 0
    c.proc = _DoneProc()
    c.lines = [(1.0, _line(1000)), (10.00, _line(1965)), (10.08, _line(1950)), (20.0, _line(1000))]
    c.mark(10.03, 10.04)
    r = c.stop()
    assert r["samples"] == 2 and r["sm_mhz"] == np.median([1965, 1950])


def test_clock_sampler_without_nvidia_smi():
    b = _bench()
    c = b.ClockSampler(0)
    r = c.stop()
    assert r["sm_mhz"] is None and r["reasons"] == ["nvidia-smi unavailable"]


def test_angle_chunks_partition_the_grid_across_ranks():
    b = _bench()
    grid = np.arange(100 * 3, dtype=float).reshape(100, 3)
    seen = []
    for s in range(2):
        for rank in range(4):
            e, start = b.chunk(grid, s, 4, rank, 10)
            assert e.shape == (10, 3) and start == ((s * 4 + rank) * 10) % 100
            seen.extend(range(start, start + 10))
    # two steps of four ranks cover 80 distinct triplets, no overlap
    assert len(set(seen)) == 80
    # past the end of the grid the chunks wrap around
    e, start = b.chunk(grid, 3, 4, 3, 10)
    assert start == 50 and np.array_equal(e[:, 0], grid[50:60, 0])
    e, _ = b.chunk(grid, 0, 1, 0, 120)
    assert np.array_equal(e[100:, 0], grid[:20, 0])
