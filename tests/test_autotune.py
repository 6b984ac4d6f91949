"""SSSP bucket-width autotuner: cache keys, cache hits and misses (CPU, with
a stand-in device graph), and on the GPU that tuning never changes results."""
import numpy as np
import pytest

from fastapsp_b200 import autotune


class FakeGraph:
    def __init__(self, best_index, dtype=0, mean_w=50.0):
        self.dtype = dtype
        self._mw = mean_w
        self.best_index = best_index
        self.params = {}
        self.tuned = 0

    def mean_weight(self):
        return self._mw

    def set_param(self, k, v):
        self.params[k] = v

    def tune_sssp(self, deltas, sample=0):
        self.tuned += 1
        ms = np.full(len(deltas), 10.0, np.float32)
        ms[self.best_index] = 1.0
        self.params["sssp_delta"] = deltas[self.best_index]
        return deltas[self.best_index], ms


def test_bucket_key_rounds_to_powers_of_two():
    vn = [0, 900, 880, 910]
    bn = [0, 5, 4, 6]
    assert autotune.bucket_key(vn, bn, 0) == "i32:nsub~2^10:nbdy~2^3"
    assert autotune.bucket_key(vn, bn, 1).startswith("f32:")


def test_tune_then_cache_hit(tmp_path):
    path = str(tmp_path / "tune.json")
    vn, bn = [0, 1000, 1024], [0, 170, 160]
    g = FakeGraph(best_index=2, mean_w=50.0)
    e = autotune.tune_sssp(g, vn, bn, path=path)
    assert not e["cached"] and e["factor"] == autotune.FACTORS[2] and g.tuned == 1
    assert e["delta"] == pytest.approx(autotune.FACTORS[2] * 50.0)
    g2 = FakeGraph(best_index=0, mean_w=10.0)      # same bucket, other weight scale
    e2 = autotune.tune_sssp(g2, vn, bn, path=path)
    assert e2["cached"] and g2.tuned == 0
    assert g2.params["sssp_delta"] == pytest.approx(autotune.FACTORS[2] * 10.0)
    e3 = autotune.tune_sssp(g2, vn, bn, path=path, force=True)
    assert not e3["cached"] and g2.tuned == 1


def test_bellman_ford_winner_is_cached_as_none(tmp_path):
    path = str(tmp_path / "tune.json")
    g = FakeGraph(best_index=len(autotune.FACTORS))
    e = autotune.tune_sssp(g, [0, 100], [0, 3], path=path)
    assert e["factor"] is None and e["delta"] == 1e9
    g2 = FakeGraph(best_index=0)
    autotune.tune_sssp(g2, [0, 100], [0, 3], path=path)
    assert g2.params["sssp_delta"] == 1e9


@pytest.mark.gpu
def test_tuning_keeps_results_bit_exact(cuda_ok, tmp_path):
    from conftest import load_golden
    from fastapsp_b200 import FAP_MODE_BATCHED, Context, DeviceGraph
    case = load_golden("grid64_k8")
    ctx = Context(0)
    ro, col, w = case["row_offset"], case["col_val"], case["weight"]
    dg = DeviceGraph(ctx, ro, col[:ro[-1]], w[:ro[-1]])
    dg.set_parts(case["K"], case["graph_id"], case["st2ed"], case["ver_num"],
                 case["ver_offset"], case["bdy_num"])
    e = autotune.tune_sssp(dg, case["ver_num"], case["bdy_num"], path=str(tmp_path / "t.json"))
    assert len(e["ms"]) == len(autotune.FACTORS) + 1 and min(e["ms"]) > 0
    dg.solve(mode=FAP_MODE_BATCHED)
    cs = np.concatenate([dg.block_checksums(p) for p in range(1, case["K"] + 1)])
    np.testing.assert_array_equal(cs, case["row_checksums"])


class FakeSolveGraph:
    """Stand-in device graph whose step time depends on the parameters."""

    def __init__(self, dtype, best):
        self.dtype = dtype
        self.best = best
        self.params = {}

    def set_param(self, k, v):
        self.params[k] = v

    def step(self):
        cur = {k: self.params.get(k) for k in self.best}
        thin_penalty = 0.5 if self.params.get("thin_max_b", 16) != self.best.get("thin_max_b", 16) else 0.0
        return (1.0 if cur == self.best else 5.0) + thin_penalty


@pytest.mark.parametrize("dtype,best", [(0, {"minplus_pack16": 1, "floyd_queue": 0}),
                                        (1, {"minplus_pack16": 0, "floyd_queue": 1})])
def test_tune_solve_picks_the_fastest_and_caches_it(tmp_path, dtype, best):
    path = str(tmp_path / "tune.json")
    vn, bn = [0, 1000, 1024], [0, 170, 160]
    g = FakeSolveGraph(dtype, best)
    out = autotune.tune_solve(g, vn, bn, g.step, path=path)
    assert out["params"] == best and not out["cached"]
    assert g.params == best
    # float32 graphs only time the Floyd form (packing applies to int32)
    assert len(out["candidates"]) == (4 if dtype == 0 else 2)
    g2 = FakeSolveGraph(dtype, best)
    out2 = autotune.tune_solve(g2, vn, bn, lambda: pytest.fail("timed again"), path=path)
    assert out2["cached"] and g2.params == best


def test_tune_solve_thin_threshold_second_pass(tmp_path):
    """Parts with 5..16 boundary vertices: the thin-kernel threshold is tuned
    after the arithmetic and Floyd form, from the best of those."""
    path = str(tmp_path / "tune.json")
    vn, bn = [0, 900, 910, 905], [0, 6, 9, 12]
    best = {"minplus_pack16": 1, "floyd_queue": 1, "thin_max_b": 8}
    g = FakeSolveGraph(0, best)
    out = autotune.tune_solve(g, vn, bn, g.step, path=path)
    assert out["params"] == best and g.params["thin_max_b"] == 8
    assert len(out["candidates"]) == 4 + 2
