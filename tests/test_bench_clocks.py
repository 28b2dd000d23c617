"""bench.py's host helpers, without a GPU.

The clock sampler: nvidia-smi runs from before the warm-up steps, and only
the samples whose timestamps fall inside the timed region are reported (all
of them when none does); the parser is checked on lines in nvidia-smi's CSV
format (timestamp first). The certificate writer that the CLI leg compares
byte for byte: checked against the committed certificates."""
import datetime
import importlib.util
import os
import tempfile

from conftest import REPO


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _Done:
    def terminate(self):
        pass

    def wait(self, timeout):
        pass


def _sampler(mod, lines, t0):
    c = mod.ClockSampler.__new__(mod.ClockSampler)
    c.path = tempfile.mktemp(suffix=".csv")
    with open(c.path, "w") as f:
        f.write("".join(lines))
    c.p = _Done()
    c.t0 = t0
    return c


def _line(ts, sm, reasons=("Not Active",) * 4):
    stamp = ts.strftime("%Y/%m/%d %H:%M:%S.") + "%03d" % (ts.microsecond // 1000)
    return f"{stamp}, 0, {sm}, 1965, 700.0, 0x0, " + ", ".join(reasons) + "\n"


def test_only_timed_region_samples_are_kept():
    mod = _bench()
    now = datetime.datetime.now()
    early = now - datetime.timedelta(seconds=10)
    lines = [_line(early, 1200, ("Not Active", "Active", "Not Active", "Not Active")),
             _line(now, 1965), _line(now, 1965, ("Not Active", "Not Active", "Not Active", "Active"))]
    r = _sampler(mod, lines, now - datetime.timedelta(seconds=1)).stop()
    assert r["samples_in_timed_region"] == 2 and r["samples"] == 2
    assert r["sm_mhz"] == 1965.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == ["sw_power_cap"]  # the early hw_thermal_slowdown sample is outside


def test_all_samples_when_none_is_inside():
    mod = _bench()
    early = datetime.datetime.now() - datetime.timedelta(seconds=10)
    r = _sampler(mod, [_line(early, 1800)], datetime.datetime.now()).stop()
    assert r["samples_in_timed_region"] == 0 and r["samples"] == 1 and r["sm_mhz"] == 1800.0


def test_certificate_text_matches_golden_files():
    """bench.py compares the CLI's certificate bytes with a text it writes
    from its own linking numbers: that writer reproduces the committed
    certificates from their entries (pairs in either order, values off the
    integer, zeros dropped)."""
    import glob

    import numpy as np

    mod = _bench()
    paths = sorted(glob.glob(os.path.join(REPO, "tests", "golden", "certificates", "*.txt")))
    assert paths
    rng = np.random.default_rng(5)
    for p in paths:
        text = open(p).read()
        lines = text.strip().splitlines()
        ncurves = int(lines[0])
        rows = [tuple(int(x) for x in ln.split(",")) for ln in lines[1:]]
        pairs = [(j, i) if k % 2 else (i, j) for k, (i, j, _) in enumerate(rows)]
        lk = [v + rng.uniform(-0.2, 0.2) for (_, _, v) in rows]
        # Pairs that round to zero are not written.
        pairs += [(0, 1), (2, 1)]
        lk += [0.1, -0.2]
        order = rng.permutation(len(pairs))
        got = mod.certificate_text(ncurves, np.array(pairs, dtype=np.int64).reshape(-1, 2)[order],
                                   np.array(lk)[order])
        assert got == text, p
