"""Host-side pieces of bench.py, on the CPU: the clock record taken during
the timed region (median SM clock, maximum clock, active slowdown reasons,
only the samples inside the window) from an nvidia-smi CSV, and the
whole-job throughput."""
import datetime
import os
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


class _Done:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _clocks_from(rows):
    import bench
    c = bench.Clocks.__new__(bench.Clocks)
    c.p = _Done()
    c.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    for r in rows:
        c.f.write(", ".join(r) + "\n")
    c.f.flush()
    return c


def _ts(t):
    return datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]


def test_clocks_window_median_and_reasons():
    t0 = 1_700_000_000.0
    idle = ["Not Active"] * 4
    rows = [
        [_ts(t0 - 5), "345", "1965", "120.0", "0x0"] + idle,            # before the window
        [_ts(t0 + 0.1), "1965", "1965", "700.0", "0x0"] + idle,
        [_ts(t0 + 0.2), "1950", "1965", "900.0", "0x4"] + ["Not Active"] * 3 + ["Active"],
        [_ts(t0 + 0.3), "1965", "1965", "950.0", "0x0"] + idle,
        [_ts(t0 + 9), "210", "1965", "100.0", "0x0"] + ["Active"] + ["Not Active"] * 3,   # after
    ]
    c = _clocks_from(rows)
    r = c.stop(t0, t0 + 1.0)
    assert r["samples"] == 3
    assert r["sm_mhz"] == 1965.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == ["sw_power_cap"]          # hw_slowdown fell outside the window


def test_clocks_reject_reason_seen_inside_window():
    t0 = 1_700_000_000.0
    rows = [[_ts(t0 + 0.1), "1200", "1965", "990.0", "0x8"] + ["Not Active", "Active", "Not Active", "Not Active"]]
    r = _clocks_from(rows).stop(t0, t0 + 1.0)
    assert r["reasons"] == ["hw_thermal_slowdown"] and r["sm_mhz"] == 1200.0


def test_throughput_is_whole_job_on_the_slowest_rank():
    import bench
    # 4 replicas of 12.648 Mpts, 10 steps, slowest rank 36 ms
    assert abs(bench.throughput(4, 12.648, 10, 36.0) - 4 * 12.648 * 10 / 0.036) < 1e-9


def test_bench_functions_resolve_their_globals():
    """Every global name a function of bench.py reads is defined at module
    level or a builtin (a function lost in an edit fails here, not on a GPU)."""
    import builtins
    import symtable
    path = os.path.join(ROOT, "bench.py")
    top = symtable.symtable(open(path).read(), path, "exec")
    defined = {s.get_name() for s in top.get_symbols() if s.is_assigned() or s.is_imported()}
    missing = []

    def walk(t):
        for ch in t.get_children():
            for s in ch.get_symbols():
                name = s.get_name()
                if s.is_global() and s.is_referenced() and name not in defined and not hasattr(builtins, name):
                    missing.append((ch.get_name(), name))
            walk(ch)

    walk(top)
    assert not missing, missing
