"""Host-side pieces of bench.py that need no GPU: the clock sampler keeps
only the samples taken inside the timed region (and reports throttle
reasons seen there), the default run keeps at least 3 warm-up steps, and
the reference arm prints its contract line from rank 0 only."""
import datetime
import importlib.util
import os
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _Done:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        pass

    def kill(self):
        pass


def _sample_line(t, sm, power_cap):
    ts = datetime.datetime.fromtimestamp(t).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    cap = "Active" if power_cap else "Not Active"
    return (f"0, {sm}, 1965, 600.0, 0x0, Not Active, Not Active, Not Active, {cap}, {ts}\n")


def test_clock_samples_are_kept_to_the_timed_region():
    b = _bench()
    c = b.ClockSampler(0)
    fd, c.path = tempfile.mkstemp(suffix=".csv")
    os.close(fd)
    now = time.time()
    with open(c.path, "w") as f:
        f.write(_sample_line(now - 2.0, 900, True))     # before: throttled, not counted
        f.write(_sample_line(now + 0.10, 1965, False))
        f.write(_sample_line(now + 0.20, 1950, False))
        f.write(_sample_line(now + 9.0, 600, True))      # after: not counted
    c.proc = _Done()
    c.mark(now, now + 0.5)
    out = c.stop()
    assert out["samples"] == 2 and out["window"] == "timed region"
    assert out["sm_mhz"] == 1957.5 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == []


def test_clock_samples_without_a_window_use_every_line():
    b = _bench()
    c = b.ClockSampler(0)
    fd, c.path = tempfile.mkstemp(suffix=".csv")
    os.close(fd)
    now = time.time()
    with open(c.path, "w") as f:
        f.write(_sample_line(now, 1800, True))
    c.proc = _Done()
    out = c.stop()
    assert out["samples"] == 1 and out["reasons"] == ["sw_power_cap"]


def test_default_run_has_three_warmup_steps(monkeypatch):
    b = _bench()
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    args = b.parse_args()
    assert args.warmup >= 3 and args.steps >= 1 and args.gpus == 1


def _run_bench(args, env_extra=None):
    import json
    import subprocess
    env = dict(os.environ)
    env.update(env_extra or {})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    return [json.loads(ln) for ln in lines]


def test_reference_arm_prints_one_contract_line():
    """`bench.py --impl reference` times the reference's CPU path on the
    host (no GPU) and prints one JSON line with the contract's keys."""
    out = _run_bench(["--impl", "reference", "--workload", "grid64", "--steps", "1", "--warmup", "0"])
    assert len(out) == 1
    line = out[0]
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "entries/s"
    assert line["higher_is_better"] is True and line["steps"] == 1 and line["n_gpus"] == 1
    assert line["config"]["workload"] == "grid64"
    cb = line["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    # the reference arm builds its workload with the generator alone and lets
    # the reference binary partition it: the product library stays unloaded
    assert line["product_library_loaded"] is False
    assert {"parallelism", "l2", "part_size", "boundary"} <= set(line["config"])


def test_reference_partition_matches_the_product():
    """The reference arm describes the workload from the reference binary's
    own preprocessing; on an undirected workload it equals the product's."""
    b = _bench()
    from fastapsp_b200 import workloads
    from oracle import oracle as O
    if not O.ref_available():
        import pytest
        pytest.skip("reference binary not built")
    wl = workloads.load("grid64")
    with tempfile.TemporaryDirectory() as tmp:
        meta = b.reference_partition(wl, tmp)
    assert b.describe_meta(wl.name, wl.K, wl.edges.directed, meta) == wl.describe()
    import numpy as np
    assert np.array_equal(meta.st2ed, wl.graph.getMapping())


def test_reference_arm_runs_on_rank_zero_only():
    out = _run_bench(["--impl", "reference", "--workload", "grid64", "--steps", "1", "--warmup", "0"],
                     {"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert out == []
