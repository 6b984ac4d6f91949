#!/usr/bin/env python
"""Benchmark of the per-subgraph APSP solve path on B200.

    python bench.py [--gpus N --steps K --warmup W] [--impl fap|reference]

One step = one full APSP solve of the workload (every part's SSSP, Floyd and
min-plus; every distance entry written to HBM).  Default workload: the
114,599-vertex road-shaped graph (integer weights 1..1000), K=128 parts.

Arms
  fap (default)  the CUDA path.  `value` = APSP entries/s of the batched form
                 with inputs resident in HBM, timed with CUDA events on the
                 library's stream (max over ranks); `plain` = the same for the
                 one-launch-sequence-per-part form; `e2e` = the public API with
                 host inputs and every block read back to pinned host memory.
  reference      the reference's own CPU path (oracle/_ref/fap_ref built from
                 the reference sources; the C restatement when that binary is
                 absent) on this host's cores, one process per core like the
                 reference's MPI driver, each step a bounded sample of parts.

With N>1 (torchrun) the parts are sharded across ranks (no data-path
collective; the reference's MPI task split); rank 0 prints the JSON line.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

# Load every kernel when the context is created, so that no timed region
# pays a kernel's first-launch module load.
os.environ.setdefault("CUDA_MODULE_LOADING", "EAGER")

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "APSP entries/sec, batched vs plain form on 1 B200 (bit-exact int32); p50/p99 latency"
UNIT = "entries/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["fap", "reference"], default="fap")
    ap.add_argument("--workload", default="road114k")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-procs", type=int, default=0, help="0 = min(cores, memory bound)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-stream measurement")
    ap.add_argument("--stage1", type=int, default=0, choices=[0, 1, 2],
                    help="stage 1 form: 0 automatic, 1 SSSP, 2 boundary graph")
    ap.add_argument("--sssp-form", type=int, default=0, choices=[0, 1, 2],
                    help="SSSP form of stage 1: 0 automatic, 1 frontier, 2 tiled Bellman-Ford")
    ap.add_argument("--bgraph-form", type=int, default=0, choices=[0, 1, 2],
                    help="boundary-graph closure: 0 by size, 1 Floyd, 2 Bellman-Ford + tiled expansion")
    ap.add_argument("--no-tune-solve", action="store_true",
                    help="keep the default min-plus arithmetic and Floyd form (no timing of the candidates)")
    ap.add_argument("--no-queue", action="store_true",
                    help="batched Floyd as three launches per pivot block instead of the work queue")
    ap.add_argument("--no-pack16", action="store_true",
                    help="min-plus tiles in int32 only (no packed 16-bit tiles)")
    ap.add_argument("--no-prepack", action="store_true",
                    help="packed min-plus tiles convert their int32 stages in shared memory instead of "
                         "reading operands packed once per solve")
    ap.add_argument("--no-stage-cache", action="store_true",
                    help="grouped jobs: run stages 1-2 per group instead of once for all parts")
    ap.add_argument("--cache-only", action="store_true",
                    help="time only stages 1-2 of every part (the resident cache build), no output matrix")
    ap.add_argument("--paths", action="store_true",
                    help="also time batched solves that produce predecessor matrices")
    ap.add_argument("--extra", default=",".join(EXTRA_WORKLOADS),
                    help="further workloads timed after the headline one (comma list, '' for none)")
    ap.add_argument("--extra-steps", type=int, default=2)
    ap.add_argument("--extra-plain-steps", type=int, default=1,
                    help="plain-form steps (one launch sequence per part) timed for each further workload")
    ap.add_argument("--extra-warmup", type=int, default=3)
    ap.add_argument("--extra-parity-parts", type=int, default=2,
                    help="parts of each further workload checked against the reference binary")
    ap.add_argument("--serve-graphs", type=int, default=32)
    ap.add_argument("--serve-burst", type=int, default=1024,
                    help="requests of the closed-loop run that measures capacity")
    ap.add_argument("--serve-seconds", type=float, default=4.0,
                    help="arrival window of each offered-load run")
    ap.add_argument("--serve-batch-rows", type=int, default=0,
                    help="output rows per batch (0: memory budget only)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic(workload, kernel):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(workload, {}).get(kernel)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,timestamp")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None
        self.window = None  # (start, stop) wall times of the timed region

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # nvidia-smi takes a moment to start: wait (bounded) for its first sample
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def mark(self, start, stop):
        """Wall times of the timed region: only samples inside it count."""
        self.window = (start, stop)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 10:
                    continue
                try:
                    row = (None, float(parts[1]), float(parts[2]), parts[5:9])
                except ValueError:
                    continue
                try:
                    t = datetime.datetime.strptime(parts[9], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                    row = (t,) + row[1:]
                except ValueError:
                    pass
                rows.append(row)
        os.unlink(self.path)
        inside = [r for r in rows if self.window and r[0] is not None
                  and self.window[0] - 0.05 <= r[0] <= self.window[1] + 0.05]
        use = inside or rows
        sm = [r[1] for r in use]
        smax = [r[2] for r in use]
        reasons = set()
        for r in use:
            for nm, v in zip(names, r[3]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm),
                "window": "timed region" if inside else "around the timed region (none inside)"}


def _jsonable(o):
    if isinstance(o, (np.floating,)):
        return float(o)
    if isinstance(o, (np.integer,)):
        return int(o)
    if isinstance(o, np.ndarray):
        return o.tolist()
    raise TypeError(type(o).__name__)


def emit(line):
    print(json.dumps(line, default=_jsonable), flush=True)


def log(msg):
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


# ---------------------------------------------------------------------------
# CPU baseline: the reference's CPU path, one process per core
# ---------------------------------------------------------------------------
def cpu_procs(requested):
    cores = os.cpu_count() or 1
    avail_gb = 8.0
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail_gb = int(line.split()[1]) / 1e6
    except OSError:
        pass
    cap = max(1, int(avail_gb * 0.5 / 1.0))   # ~1 GB per process (block + path)
    p = min(cores, cap, 64)
    if requested:
        p = min(p, requested)
    return max(1, p)


def run_reference_sample(wl, parts_per_proc, procs, timeout=900, extra=None, partition_file=None,
                         threads=1):
    """Runs the reference CPU path on `procs` concurrent processes, process i
    solving parts_per_proc[i] in order (extra[i]: more arguments of process
    i, e.g. output files; partition_file: a shared partition in place of the
    reference's METIS call).  Returns (kind, per-process list of
    (part, rows, entries, seconds))."""
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    if partition_file:
        env["FAP_PARTITION_FILE"] = os.path.abspath(partition_file)
    if kind == "reference":
        cmds = [[O.REF_BIN, "--dir", wl.root, "-f", wl.name, "-k", str(wl.K),
                 "-direct", str(int(wl.edges.directed)), "-weight", str(int(wl.edges.weighted)),
                 "--parts", ",".join(map(str, pp)), "--quiet"] + list((extra or {}).get(i, []))
                for i, pp in enumerate(parts_per_proc)]
    else:
        script = os.path.join(ROOT, "oracle", "port_cli.py")
        cmds = [[sys.executable, script, "--dir", wl.root, "-f", wl.name, "-k", str(wl.K),
                 "-direct", str(int(wl.edges.directed)), "-weight", str(int(wl.edges.weighted)),
                 "--parts", ",".join(map(str, pp))] for pp in parts_per_proc]
    ps = [subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env)
          for c in cmds]
    out = []
    for p in ps:
        so, se = p.communicate(timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"CPU baseline process failed: {se[-500:]}")
        rec = [json.loads(x) for x in so.splitlines() if x.startswith("{")]
        out.append([(r["part"], r["rows"], r["entries"], r["seconds"]) for r in rec
                    if r.get("event") == "part"])
    return kind, out


PARITY_FLOAT_PARTS = 4   # float32 workloads: whole blocks compared for this many parts
FLOAT_RTOL = 1e-5        # float32 bar: |d - ref| <= 1e-5 |ref|, reachability exact


def gpu_parity_blocks(dg, groups, parts, dtype, staged, mode):
    """What the GPU produced for the parity sample: per-row checksums of each
    part's block (int32) or the blocks themselves (float32, the first
    PARITY_FLOAT_PARTS parts).  Blocks of the timed run are still resident
    when the job is one group; otherwise the groups holding sampled parts
    are solved again (untimed) the way the timed loop solves them."""
    from fastapsp_b200 import FAP_DTYPE_F32
    want = set(parts if dtype == 0 else parts[:PARITY_FLOAT_PARTS])
    out = {}
    for grp in groups:
        hit = [p for p in grp if p in want]
        if not hit:
            continue
        if len(groups) > 1:
            dg.solve(grp, mode)
        for p in hit:
            out[p] = (dg.block_checksums(p) if dtype == 0
                      else dg.copy_block(p, out_dtype=FAP_DTYPE_F32))
    dg.check()
    return out


def compare_parity(wl, gpu, ref_files, dtype, st2ed, ref_meta):
    """Compares the GPU's blocks of the sampled parts with the reference
    binary's output for the same parts under the same partition."""
    rows = mism = 0
    worst = 0.0
    reach_mism = 0
    n = wl.n
    for p, f in ref_files.items():
        if p not in gpu:
            continue
        if dtype == 0:
            ref = np.fromfile(f, dtype=np.uint64)
            got = gpu[p]
            rows += int(got.size)
            mism += int(got.size) if ref.size != got.size else int((ref != got).sum())
        else:
            ref = np.fromfile(f, dtype=np.float32).reshape(-1, n)
            got = gpu[p]
            rows += int(got.shape[0])
            inf_r, inf_g = ref >= np.float32(1e8), got >= np.float32(1e8)
            reach_mism += int((inf_r != inf_g).sum())
            fin = ~inf_r & ~inf_g
            err = np.abs(got[fin].astype(np.float64) - ref[fin]) / np.maximum(np.abs(ref[fin]), 1e-30)
            e = float(err.max()) if err.size else 0.0
            worst = max(worst, e)
            mism += int((err > FLOAT_RTOL).sum()) + int((inf_r != inf_g).sum())
    res = {"config": wl.name, "parts": len([p for p in ref_files if p in gpu]), "rows": rows,
           "mismatches": mism,
           "st2ed_equal": (bool(np.array_equal(ref_meta.st2ed, st2ed))
                           if ref_meta is not None else None),
           "partition": "the GPU run's partition given to the reference binary (FAP_PARTITION_FILE)"}
    if dtype == 0:
        res["rule"] = "bit-exact int32: per-row checksums sum_j uint32(d[r][j])*(2j+1) mod 2^64"
        res["mismatches_unit"] = "rows"
    else:
        res["rule"] = f"float32: |d - ref| <= {FLOAT_RTOL} |ref|, reachability exact"
        res["mismatches_unit"] = "entries"
        res["max_rel_err"] = worst
        res["reachability_mismatches"] = reach_mism
    return res


def sample_parts(K, count, seed):
    rng = np.random.default_rng(seed)
    return [int(x) + 1 for x in rng.permutation(K)[:count]]


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def reference_partition(wf, workdir):
    """The reference binary's own host preprocessing of the workload file
    (MatrixMarket reader, METIS, findBoundry, sort_and_encode): its CSR,
    partition and renumbering, read back from `fap_ref --parts none --meta`.
    Returns None when the reference binary is absent."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    meta = os.path.join(workdir, "ref_meta.bin")
    O.run_ref(wf.root, wf.name, wf.edges.directed, wf.edges.weighted, wf.K, parts="none",
              meta_out=meta, threads=1, timeout=900)
    m = O.read_meta(meta)
    os.unlink(meta)
    return m


def describe_meta(name, K, directed, m):
    """The workload description of `Workload.describe`, from the reference's
    own preprocessing."""
    vn, bn = m.ver_num[1:], m.bdy_num[1:]
    return {"workload": name, "n": int(m.n), "arcs": int(m.row_offset[-1]), "K": int(K),
            "directed": bool(directed), "avg_degree": round(float(m.row_offset[-1]) / m.n, 3),
            "part_size": [int(vn.min()), int(np.median(vn)), int(vn.max())],
            "boundary": [int(bn.min()), int(np.median(bn)), int(bn.max()), int(bn.sum())]}


def common_config(desc, n_gpus):
    """The `config` both arms print: the workload's description, the
    parallelism and what keeps L2 from serving the timed steps."""
    n = int(desc["n"])
    return {**desc, "parallelism": f"parts sharded x{n_gpus}",
            "l2": (f"outputs larger than L2: each step writes {4 * n * n / 1e9:.1f} GB of "
                   "distances; the GPU arm also writes a 256 MB buffer between timed steps, "
                   "outside the events")}


def product_library_loaded():
    """Whether this process has mapped the product's shared library."""
    try:
        with open("/proc/self/maps") as f:
            return any("libfap_b200.so" in ln for ln in f)
    except OSError:
        return None


def main_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    # Only the seeded generator and the MatrixMarket writer run here: the
    # reference binary reads the file, partitions it with METIS and renumbers
    # it itself, so this process never loads the product's library.
    from fastapsp_b200 import workloads
    wf = workloads.write(args.workload)
    with tempfile.TemporaryDirectory() as tmp:
        meta = reference_partition(wf, tmp)
    if meta is not None:
        config = common_config(describe_meta(wf.name, wf.K, wf.edges.directed, meta), args.gpus)
    else:
        config = common_config({"workload": wf.name, "n": wf.n, "K": wf.K,
                                "directed": wf.edges.directed}, args.gpus)
    P = cpu_procs(args.cpu_procs)
    steps = args.warmup + args.steps
    need = P * steps
    order = [int(x) + 1 for x in np.random.default_rng(7).permutation(wf.K)]
    order = (order * (need // wf.K + 1))[:need]
    per = [order[i::P] for i in range(P)]
    kind, res = run_reference_sample(wf, per, P)
    tot_entries, tot_time, step_ms = 0, 0.0, []
    for s in range(args.warmup, steps):
        ent = sum(r[s][2] for r in res)
        sec = max(r[s][3] for r in res)
        tot_entries += ent
        tot_time += sec
        step_ms.append(sec * 1e3)
    value = tot_entries / tot_time
    sample = (f"{args.steps} timed steps x {P} processes x 1 part "
              f"({wf.name}, K={wf.K}); step time = slowest process")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": float(np.mean(step_ms)), "higher_is_better": True,
        "impl": "reference", "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": config,
        "solve": {"mode": "reference CPU path (oracle/_ref/fap_ref: the reference's fap.cpp, "
                          "fapGraph::run per part)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": P, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "product_library_loaded": product_library_loaded(),
    }
    emit(line)


# ---------------------------------------------------------------------------
# fap arm
# ---------------------------------------------------------------------------
def run_serving(args, device):
    """Serving stream: Poisson arrivals of solveSubGraph / distance-row
    requests over resident random-geometric graphs, answered by the native
    serving loop (fap_server_*).  Capacity is measured in a closed loop (64
    requests in flight); then requests arrive at 25/50/90% of it.  Each
    request returns per-row checksums (its distances stay in HBM)."""
    from fastapsp_b200 import workloads
    from fastapsp_b200.serve import Server

    t0 = time.perf_counter()
    gs = workloads.load_serve_stream(args.serve_graphs)
    log(f"serving stream: {len(gs)} graphs built in {time.perf_counter() - t0:.1f} s")
    import torch
    free_b = torch.cuda.mem_get_info()[0]
    srv = Server(device, budget_bytes=0.6 * free_b, max_batch_rows=args.serve_batch_rows)
    info = []
    for g in gs:
        idx = srv.add_graph(g.graph)
        vn = g.graph.partInfo()[0]
        info.append((idx, g.n, g.K, vn))
    rng = np.random.default_rng(23)

    def draw():
        gi, n, K, vn = info[int(rng.integers(len(info)))]
        if rng.random() < 0.8:
            return ("sub", gi, int(rng.integers(1, K + 1)))
        cnt = int(round(np.exp(rng.uniform(np.log(100), np.log(10000)))))
        return ("rows", gi, rng.integers(0, n, min(cnt, n)).astype(np.int32))

    def submit(req):
        if req[0] == "sub":
            return srv.submit_subgraph(req[1], req[2], distances=False, checksums=True)
        return srv.submit_rows(req[1], req[2], distances=False, checksums=True)

    def finish(handles, kinds=None):
        """Waits for the handles; returns per-kind latency percentiles."""
        srv.drain()
        lat = {"sub": [], "rows": []}
        for i, h in enumerate(handles):
            if h.wait(0) != 2:
                raise RuntimeError(f"serving request failed: {h.info()}")
            if kinds is not None:
                lat[kinds[i]].append(h.info()["latency_ms"])
            h.forget()
        return {k: {"requests": len(v), "p50_ms": float(np.percentile(v, 50)) if v else None,
                    "p99_ms": float(np.percentile(v, 99)) if v else None} for k, v in lat.items()}

    # warm-up: one request of each kind per graph (resident caches, batch buffers)
    finish([srv.submit_subgraph(i, 1, distances=False, checksums=True) for i, *_ in info] +
           [srv.submit_rows(i, np.arange(100, dtype=np.int32) % n, distances=False, checksums=True)
            for i, n, *_ in info])
    warm = srv.stats()
    log(f"serving warm-up: {warm.cache_builds} caches built, {warm.busy_ms:.1f} ms device time")
    window = 64

    def closed_loop(reqs):
        t0 = time.perf_counter()
        hs, pending = [], []
        for r in reqs:
            if len(pending) >= window:
                pending.pop(0).wait()
            h = submit(r)
            hs.append(h)
            pending.append(h)
        by_kind = finish(hs, [r[0] for r in reqs])
        return by_kind, time.perf_counter() - t0

    # warm-up of the mixed stream itself (every kernel shape it uses, batch
    # buffers at their working sizes), untimed
    closed_loop([draw() for _ in range(max(64, args.serve_burst))])
    # capacity: closed loop, a window of 64 requests in flight, measured twice;
    # the lower figure sets the offered loads, so that "90%" is not an overload
    caps = []
    for _ in range(2):
        srv.reset_stats()
        reqs = [draw() for _ in range(args.serve_burst)]
        by_kind, burst_s = closed_loop(reqs)
        caps.append((len(reqs) / burst_s, burst_s, by_kind, srv.stats()))
    cap_rps, burst_s, by_kind, st = min(caps, key=lambda c: c[0])
    out = {"graphs": len(gs),
           "n": [min(g.n for g in gs), max(g.n for g in gs)],
           "K": sorted({g.K for g in gs}),
           "part_rows": [int(min(x[3][1:].min() for x in info)), int(max(x[3][1:].max() for x in info))],
           "mix": "80% solveSubGraph (uniform graph, uniform part), 20% distance rows "
                  "(100-10,000 sources, log-uniform); per-row checksums returned",
           "budget_bytes": int(0.6 * free_b),
           "capacity": {"requests_s": cap_rps, "runs_requests_s": [c[0] for c in caps],
                        "entries_s": st.entries / burst_s,
                        "requests": len(reqs), "window": window, "batches": st.batches,
                        "resident_hits": st.resident_hits, "p50_ms": st.p50_ms, "p99_ms": st.p99_ms,
                        "by_kind": by_kind, "device_busy_frac": st.busy_ms * 1e-3 / burst_s,
                        "worker_host_max_ms": {k: round(v, 3) for k, v in st.host_max_ms.items()}},
           "warmup_cache_builds": warm.cache_builds,
           "loads": []}
    log(f"serving capacity {cap_rps:.1f} req/s (runs {[round(c[0], 1) for c in caps]}), "
        f"{st.entries / burst_s:.4g} entries/s (closed loop, {window} in flight)")
    for frac in (0.25, 0.5, 0.9):
        rate = frac * cap_rps
        count = int(min(max(32, rate * args.serve_seconds), 2 * args.serve_burst))
        reqs = [draw() for _ in range(count)]
        gaps = rng.exponential(1.0 / rate, count)
        srv.reset_stats()
        hs = []
        t0 = time.perf_counter()
        due = t0
        for r, gap in zip(reqs, gaps):
            due += gap
            while True:
                now = time.perf_counter()
                if now >= due:
                    break
                time.sleep(min(due - now, 0.002))
            hs.append(submit(r))
        t_sub = time.perf_counter() - t0
        by_kind = finish(hs, [r[0] for r in reqs])
        wall = time.perf_counter() - t0
        st = srv.stats()
        out["loads"].append({"offered_frac": frac, "offered_requests_s": rate,
                             "requests": count, "arrival_window_s": t_sub,
                             "achieved_requests_s": count / wall, "entries_s": st.entries / wall,
                             "p50_ms": st.p50_ms, "p99_ms": st.p99_ms, "mean_ms": st.mean_ms,
                             "by_kind": by_kind,
                             "batches": st.batches, "resident_hits": st.resident_hits,
                             "peak_device_bytes": st.peak_bytes, "cache_builds": st.cache_builds,
                             "device_busy_frac": st.busy_ms * 1e-3 / wall,
                             "worker_host_max_ms": {k: round(v, 3) for k, v in st.host_max_ms.items()}})
        log(f"serving at {frac:.0%}: p50 {st.p50_ms:.2f} ms, p99 {st.p99_ms:.2f} ms, "
            f"{st.entries / wall:.4g} entries/s, {st.batches} batches; "
            f"sub p50/p99 {by_kind['sub']['p50_ms']}/{by_kind['sub']['p99_ms']}, "
            f"rows p50/p99 {by_kind['rows']['p50_ms']}/{by_kind['rows']['p99_ms']}")
    srv.close()
    return out


def run_cache_only(args, dg, stream, world):
    """Stages 1-2 of every part into the resident cache (boundary rows and
    closed Floyd matrices), without the output matrix: the profiling mode of
    stage 1 (a few GB on the device for the grid256 stand-in)."""
    import torch
    dg.cache_build()
    dg.check()
    for _ in range(args.warmup):
        dg.cache_build(rebuild=True)
    torch.cuda.synchronize()
    ms, phases = [], []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dg.cache_build(rebuild=True)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        phases.append(dg.cache_timing())
    dg.check()
    ph = np.round(np.mean(phases, 0), 3).tolist()
    log(f"cache build: {np.mean(ms):.3f} ms ({dg.stage1_name() or 'cache'}), phases {ph}")
    if int(os.environ.get("RANK", "0")) == 0:
        print(json.dumps({"mode": "cache_only", "ms_per_step": float(np.mean(ms)), "steps": args.steps,
                          "phases_ms": ph, "world": world}))


EXTRA_WORKLOADS = ("grid512", "rmat16")


def start_extra(args, name):
    """Loads a further workload on the host and starts the reference binary
    on its parity sample in the background (the reference's serial min-plus
    of a grid512 part takes minutes), so that it runs while the GPU is
    measured.  The sample: the part with the fewest boundary vertices, then
    the next ones with at least one boundary vertex."""
    from fastapsp_b200 import workloads
    from oracle import oracle as O
    t0 = time.perf_counter()
    wl = workloads.load(name)
    bn = wl.bdy_num
    order = sorted(range(1, wl.K + 1), key=lambda p: (int(bn[p]), p))
    ppart = order[:1] + [p for p in order[1:] if int(bn[p]) > 0][:max(0, args.extra_parity_parts - 1)]
    ppart = ppart[:max(0, args.extra_parity_parts)]
    job = {"wl": wl, "parts": ppart, "procs": [], "tmp": None, "files": {}, "meta": None,
           "t0": time.perf_counter(), "integral": bool(wl.edges.integral)}
    if ppart and O.ref_available():
        job["tmp"] = tempfile.TemporaryDirectory()
        tmp = job["tmp"].name
        pfile = os.path.join(tmp, "partition.bin")
        (np.asarray(wl.graph.getGraphId(), dtype=np.int64) - 1).astype(np.int32).tofile(pfile)
        job["meta"] = os.path.join(tmp, "meta.bin")
        env = dict(os.environ, OMP_NUM_THREADS=str(max(1, min(8, (os.cpu_count() or 1) // 4))),
                   FAP_PARTITION_FILE=pfile)
        for i, p in enumerate(ppart):
            f = os.path.join(tmp, f"out_{p}.bin")
            job["files"][p] = f
            cmd = [O.REF_BIN, "--dir", wl.root, "-f", wl.name, "-k", str(wl.K),
                   "-direct", str(int(wl.edges.directed)), "-weight", str(int(wl.edges.weighted)),
                   "--parts", str(p), "--quiet", "--rowsum" if job["integral"] else "--dist", f]
            if i == 0:
                cmd += ["--meta", job["meta"]]
            job["procs"].append(subprocess.Popen(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                                                 text=True, env=env))
    log(f"{name} loaded in {time.perf_counter() - t0:.1f} s: {wl.describe()}; reference started on "
        f"parts {ppart}")
    return job


def finish_extra_parity(job, gpu, dtype):
    """Waits for the reference processes of start_extra and compares."""
    from oracle import oracle as O
    if not job["procs"]:
        return {"unavailable": "reference binary absent"} if job["parts"] else None
    for pr in job["procs"]:
        _, err = pr.communicate(timeout=1800)
        if pr.returncode != 0:
            return {"unavailable": f"reference process failed: {err[-300:]}"}
    wl = job["wl"]
    parity = compare_parity(wl, gpu, job["files"], dtype, wl.graph.getMapping(), O.read_meta(job["meta"]))
    parity["parts_chosen"] = "fewest boundary vertices (one part, then parts with boundary vertices)"
    parity["parts_ids"] = job["parts"]
    parity["reference_s"] = round(time.perf_counter() - job["t0"], 2)
    job["tmp"].cleanup()
    return parity


def run_extra(args, job, ctx, relax_peak, hbm_peak, peak_kind):
    """A further workload of the same metric on one GPU: batched solves of
    every part (timed with CUDA events on the library's stream, inputs
    resident, L2 flushed between steps), its min-plus as a fraction of the
    measured relaxation peak, and parity of sampled parts against the
    reference binary under the same partition (started by start_extra)."""
    import torch

    from fastapsp_b200 import FAP_MODE_BATCHED, FAP_MODE_PLAIN, DeviceGraph, autotune
    from fastapsp_b200.sharding import group_parts_by_rows, rows_of
    wl = job["wl"]
    name = wl.name
    n = wl.n
    vn, vo, bn = wl.ver_num, wl.ver_offset, wl.bdy_num
    ro, col, w = wl.csr()
    gid = wl.graph.getGraphId()
    st2ed = wl.graph.getMapping()
    dg = DeviceGraph(ctx, ro, col, w)
    dtype = dg.dtype
    dg.set_parts(wl.K, gid, st2ed, vn, vo, bn)
    dg.set_param("minplus_pack16", 0 if args.no_pack16 else 1)
    dg.set_param("minplus_prepack", 0 if args.no_prepack else 1)
    dg.set_param("floyd_queue", 0 if args.no_queue else 1)
    ldD = (n + 127) // 128 * 128
    stream = torch.cuda.current_stream()
    mine = list(range(1, wl.K + 1))
    all_rows = rows_of(mine, vn)
    free_b = torch.cuda.mem_get_info()[0]
    budget_rows = int(0.60 * free_b / (4 * ldD))
    staged = all_rows > budget_rows
    if staged:
        dg.cache_build()
        dg.check()
        budget_rows = int(0.60 * torch.cuda.mem_get_info()[0] / (4 * ldD))
    groups = [mine] if all_rows <= budget_rows else group_parts_by_rows(mine, vn, budget_rows)
    dg.reserve(max(rows_of(g, vn) for g in groups) if len(groups) > 1 else 0)
    tuned = autotune.tune_sssp(dg, vn, bn)
    log(f"{name}: {len(groups)} group(s)")

    def step():
        if staged:
            dg.cache_build(rebuild=True)
        for grp in groups:
            dg.solve(grp, FAP_MODE_BATCHED, check_errors=False)

    def timed_first_group():
        # one stage-1-2 pass (when staged) and the first group: the choices
        # tuned affect both, and the other groups repeat the first
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        if staged:
            dg.cache_build(rebuild=True)
        dg.solve(groups[0], FAP_MODE_BATCHED, check_errors=False)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    solve_tuned = None
    if not (args.no_pack16 or args.no_queue or args.no_tune_solve):
        solve_tuned = autotune.tune_solve(dg, vn, bn, timed_first_group, reps=1)
        dg.check()
        log(f"{name}: solve form {solve_tuned['params']} ({'cached' if solve_tuned['cached'] else 'tuned'}: "
            f"{solve_tuned['ms']} ms)")

    for _ in range(args.extra_warmup):
        step()
    dg.check()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    ms, mp_ms, fl_ms = [], [], []
    for _ in range(args.extra_steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        mp = fl = 0.0
        if staged:
            dg.cache_build(rebuild=True)
        for grp in groups:
            dg.solve(grp, FAP_MODE_BATCHED, check_errors=False)
            mp += float(dg.last_timing()[3])
            fl += float(dg.last_timing()[2])
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        mp_ms.append(mp)
        fl_ms.append(fl)
    dg.check()
    # the plain form of the same job: one launch sequence per part (stage 1
    # by SSSP from that part's boundary vertices), the groups as above
    plain_ms = []
    for _ in range(max(0, args.extra_plain_steps)):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for grp in groups:
            dg.solve(grp, FAP_MODE_PLAIN, check_errors=False)
        e1.record(stream)
        e1.synchronize()
        plain_ms.append(e0.elapsed_time(e1))
    dg.check()
    del flush
    ms_step = float(np.mean(ms))
    mp_step = float(np.mean(mp_ms))
    mp_relax = float(sum(float(vn[p] - bn[p]) * float(bn[p]) * n for p in mine))
    mp_bytes = float(sum(4.0 * ((vn[p] - bn[p]) * n + (vn[p] - bn[p]) * bn[p] + bn[p] * n) for p in mine))
    # With stage 1 by SSSP and int32-only min-plus tiles (float32, or packing
    # off), the min-plus tiles run inside the Floyd work queue: the stage
    # timings then hold Floyd and min-plus together.
    form = solve_tuned["params"] if solve_tuned else {"minplus_pack16": int(not args.no_pack16),
                                                      "floyd_queue": int(not args.no_queue)}
    stage1_now = dg.stage1_name()
    mp_in_queue = (bool(form["floyd_queue"]) and stage1_now.startswith("SSSP")
                   and (dtype != 0 or not form["minplus_pack16"]))
    mp_note = None
    if mp_in_queue:
        mp_step += float(np.mean(fl_ms))
        mp_relax += float(sum(float(vn[p]) ** 3 for p in mine))
        mp_note = ("the min-plus tiles ran inside the Floyd work queue: time and relaxations of "
                   "Floyd-Warshall and min-plus together")
    a = mp_relax / (mp_step * 1e-3) / 1e9
    gpu = gpu_parity_blocks(dg, groups, job["parts"], dtype, staged, FAP_MODE_BATCHED) if job["parts"] else {}
    stage1 = dg.stage1_name()
    pk_tiles = dg.pack16_tiles()
    xk_tiles = dg.expand16_tiles()
    del dg
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    out = {
        "value": all_rows * n / (ms_step * 1e-3), "unit": UNIT, "ms_per_step": ms_step,
        "steps": args.extra_steps, "warmup": args.extra_warmup,
        "dtype": "int32" if dtype == 0 else "f32", "data": wl.data_description(),
        "config": {**wl.describe(), "groups": len(groups), "stage_cache": staged, "stage1": stage1,
                   "minplus_packed_tiles": {"packed": pk_tiles[0], "total": pk_tiles[1]},
                   "expansion_packed_tiles": {"packed": xk_tiles[0], "total": xk_tiles[1]},
                   "sssp_delta_factor": tuned["factor"],
                   "solve_form": (solve_tuned["params"] if solve_tuned else
                                  {"minplus_pack16": int(not args.no_pack16), "floyd_queue": int(not args.no_queue)}),
                   "l2": "256 MB buffer written between timed steps (outside the events); "
                         f"each step writes {4 * n * all_rows / 1e9:.1f} GB of distances"},
        "minplus": {"ms": mp_step, "relax": mp_relax, "bytes": mp_bytes, "achieved_grelax_s": a,
                    "frac_of_relax_peak": a / (relax_peak / 1e9),
                    # a packed tile relaxes two entries per instruction: with a
                    # share f of the tiles (and so of the relaxations) packed,
                    # the instructions are R (1 - f / 2)
                    "packed_tile_share": (pk_tiles[0] / pk_tiles[1]) if pk_tiles[1] else 0.0,
                    "frac_of_instruction_peak": a / (relax_peak / 1e9)
                    * (1.0 - 0.5 * ((pk_tiles[0] / pk_tiles[1]) if pk_tiles[1] else 0.0)),
                    "frac_of_hbm": mp_bytes / (mp_step * 1e-3) / 1e9 / hbm_peak,
                    "peaks": f"relaxation peak measured live (fap_measure_relax_peak, one relaxation per "
                             f"32-bit DPX instruction); HBM {peak_kind}",
                    "note": mp_note},
        "parity": None,
    }
    if plain_ms:
        pm = float(np.mean(plain_ms))
        out["plain"] = {"value": all_rows * n / (pm * 1e-3), "ms_per_step": pm, "steps": len(plain_ms)}
        out["batched_over_plain"] = pm / ms_step
    log(f"{name}: {ms_step:.1f} ms/step, {out['value']:.4g} entries/s, min-plus {mp_step:.1f} ms "
        f"({out['minplus']['frac_of_relax_peak']:.2f} of the relaxation peak)"
        + (f"; plain {float(np.mean(plain_ms)):.1f} ms/step" if plain_ms else ""))
    return out, gpu, dtype


def main_fap(args):
    import torch
    import torch.distributed as dist

    from fastapsp_b200 import FAP_DTYPE_F32, FAP_MODE_BATCHED, FAP_MODE_PLAIN, Context, DeviceGraph
    from fastapsp_b200 import workloads
    from fastapsp_b200.sharding import group_parts_by_rows, reduce_over_ranks, rows_of, shard_parts

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        # Ranks do the same work between collectives (loading the workload,
        # tuning, one timed pass); a rank that died or hangs ends the others'
        # next collective with an error after this long.
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def allmax(x):
        return reduce_over_ranks(x, "max", device="cuda")

    def allsum(x):
        return reduce_over_ranks(x, "sum", device="cuda")

    # further workloads: loaded on the host first, so that the reference's
    # parity runs of their sampled parts proceed while the GPU is measured
    extra_jobs = {}
    if rank == 0 and world == 1 and args.extra:
        for name in [x for x in args.extra.split(",") if x]:
            try:
                extra_jobs[name] = start_extra(args, name)
            except Exception as e:  # noqa: BLE001 - reported in the line, not fatal
                extra_jobs[name] = e
                log(f"{name}: {e}")

    t_load = time.perf_counter()
    wl = workloads.load(args.workload)
    log(f"workload {wl.name} loaded in {time.perf_counter() - t_load:.1f} s: {wl.describe()}")
    n = wl.n
    vn, vo, bn = wl.ver_num, wl.ver_offset, wl.bdy_num
    mine = shard_parts(vn, bn, n, world)[rank]
    my_rows = rows_of(mine, vn)
    my_entries = my_rows * n
    total_entries = allsum(my_entries)
    ro, col, w = wl.csr()
    gid = wl.graph.getGraphId()
    st2ed = wl.graph.getMapping()

    ctx = Context(local)
    ctx.use_torch_stream()
    stream = torch.cuda.current_stream()
    dg = DeviceGraph(ctx, ro, col, w)
    dtype = dg.dtype
    dg.set_parts(wl.K, gid, st2ed, vn, vo, bn)
    # Output rows that fit on the device (leaving room for the Floyd arena,
    # scratch and the e2e copy); larger jobs are produced in groups of parts.
    ldD = (n + 127) // 128 * 128
    dg.set_param("stage1", args.stage1)
    dg.set_param("sssp_form", args.sssp_form)
    dg.set_param("bgraph_form", args.bgraph_form)
    dg.set_param("minplus_pack16", 0 if args.no_pack16 else 1)
    dg.set_param("minplus_prepack", 0 if args.no_prepack else 1)
    dg.set_param("floyd_queue", 0 if args.no_queue else 1)
    if args.cache_only:
        run_cache_only(args, dg, stream, world)
        if world > 1:
            dist.destroy_process_group()
        return
    free_b = torch.cuda.mem_get_info()[0]
    budget_rows = int(0.60 * free_b / (4 * ldD))
    # A job larger than the device is produced in groups of parts.  On one
    # GPU, stages 1-2 of every part then run once per step (the resident
    # cache: boundary rows and closed Floyd matrices of all parts) and each
    # group only runs its min-plus merge from it; the cache is allocated
    # before the groups are sized.
    staged = my_rows > budget_rows and world == 1 and not args.no_stage_cache
    if staged:
        dg.cache_build()
        dg.check()
        free_b = torch.cuda.mem_get_info()[0]
        budget_rows = int(0.60 * free_b / (4 * ldD))
        log(f"stage 1-2 cache for all parts: {dg.cache_bytes()[0] / 2**30:.1f} GiB "
            f"({dg.stage1_name() or 'built'})")
    if my_rows <= budget_rows:
        groups = [mine]
        dg.reserve(0 if world == 1 else my_rows)
    else:
        groups = group_parts_by_rows(mine, vn, budget_rows)
        dg.reserve(max(rows_of(g, vn) for g in groups))
    log(f"{len(groups)} group(s) of parts; rows budget {budget_rows}")

    # N > 1: the sharded boundary-graph form when the graph takes it (each
    # rank closes its own parts locally, an NCCL all-gather exchanges their
    # boundary rows, each rank closes the boundary graph and merges its own
    # parts); otherwise each rank's partial batch takes stage 1 by SSSP
    shard = None
    if world > 1 and args.stage1 != 1 and not staged:
        from fastapsp_b200 import FapError
        from fastapsp_b200.sharding import shard_layout
        owner, elems, stride, _ = shard_layout(vn, bn, shard_parts(vn, bn, n, world))
        tdt = torch.int32 if dtype == 0 else torch.float32
        send = torch.zeros(max(stride, 1), dtype=tdt, device="cuda")
        recv = torch.zeros(world * max(stride, 1), dtype=tdt, device="cuda")
        try:
            dg.shard_begin(mine, send.data_ptr(), stride)
            shard = (owner, stride, send, recv)
        except FapError as e:
            log(f"sharded boundary-graph form not available ({e}); partial batches per rank")
        barrier()

    def solve_all(mode):
        if shard is not None and mode == FAP_MODE_BATCHED:
            owner_, stride_, send_, recv_ = shard
            dg.shard_begin(mine, send_.data_ptr(), stride_)
            dist.all_gather_into_tensor(recv_, send_)
            dg.shard_finish(recv_.data_ptr(), world, owner_, stride_)
            for grp in groups:
                dg.solve(grp, mode, check_errors=False)
            return
        if staged and mode == FAP_MODE_BATCHED:
            dg.cache_build(rebuild=True)
        for grp in groups:
            dg.solve(grp, mode, check_errors=False)
    from fastapsp_b200 import autotune
    tuned = autotune.tune_sssp(dg, vn, bn)
    log(f"SSSP delta {tuned['delta']:.6g} ({'cached' if tuned['cached'] else 'tuned'}: "
        f"{tuned['key']}, factor {tuned['factor']})")

    def timed_step():
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solve_all(FAP_MODE_BATCHED)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    solve_tuned = None
    if not (args.no_pack16 or args.no_queue or args.no_tune_solve or shard is not None):
        solve_tuned = autotune.tune_solve(dg, vn, bn, timed_step)
        dg.check()
        log(f"solve form {solve_tuned['params']} ({'cached' if solve_tuned['cached'] else 'tuned'}: "
            f"{solve_tuned['ms']} ms)")
    relax_peak = ctx.relax_peak(dtype)
    hbm_peak, peak_kind = read_peaks()

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    # ---- batched, device-resident inputs ----
    for _ in range(args.warmup):
        solve_all(FAP_MODE_BATCHED)
    dg.check()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t_timed = time.time()
    step_ms, stages = [], []
    cache_phases = []
    launches = 0
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st_step = np.zeros(5)
        if staged:
            ec = torch.cuda.Event(enable_timing=True)
            dg.cache_build(rebuild=True)
            launches += dg.last_launches()
            ec.record(stream)
        if shard is not None:
            owner_, stride_, send_, recv_ = shard
            dg.shard_begin(mine, send_.data_ptr(), stride_)
            launches += dg.last_launches()
            dist.all_gather_into_tensor(recv_, send_)
            dg.shard_finish(recv_.data_ptr(), world, owner_, stride_)
            launches += dg.last_launches()
        for grp in groups:
            dg.solve(grp, FAP_MODE_BATCHED, check_errors=False)
            if len(groups) > 1:
                st_step += dg.last_timing()
                launches += dg.last_launches()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        if len(groups) == 1:
            st_step = dg.last_timing()
            launches += dg.last_launches()
        if staged:   # the cache build holds stages 1-2 of every part
            cb = e0.elapsed_time(ec)
            ct = dg.cache_timing()
            cache_phases.append(ct)
            if "boundary graph" in dg.stage1_name():   # local closures, closure, expansion, fix-up
                st_step[0] += ct[1] + ct[2] + ct[3]
                st_step[2] += ct[0]
            else:                                       # SSSP, gather, Floyd
                st_step[0] += ct[0]
                st_step[1] += ct[1]
                st_step[2] += ct[2]
            st_step[4] += cb
        stages.append(st_step)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks.mark(t_timed, time.time())
    clk = clocks.stop()
    dg.check()
    my_ms = float(np.sum(step_ms))
    max_ms = allmax(my_ms)
    ms_per_step = max_ms / args.steps
    value = total_entries * args.steps / (max_ms * 1e-3)
    st = np.mean(np.stack(stages), 0)  # [sssp, gather, floyd, minplus, total]
    stage1_used = dg.stage1_name()

    # ---- parity sample: the timed run's blocks of the parts that the CPU
    # baseline leg below has the reference binary solve (rank 0, N=1) ----
    cpu_leg = rank == 0 and world == 1 and not args.no_cpu_baseline
    parity_parts = sample_parts(wl.K, cpu_procs(args.cpu_procs), seed=11) if cpu_leg else []
    gpu_par = (gpu_parity_blocks(dg, groups, parity_parts, dtype, staged, FAP_MODE_BATCHED)
               if parity_parts else {})
    log(f"batched: {ms_per_step:.3f} ms/step, stages {np.round(st, 3).tolist()}, "
        f"{value:.4g} entries/s")

    # ---- batched with predecessor matrices (optional) ----
    paths = None
    if args.paths and shard is None:
        try:
            dg.set_param("paths", 1)
            dg.solve(groups[0], FAP_MODE_BATCHED, check_errors=True)   # allocates P
            p_ms = []
            for _ in range(max(2, args.steps // 2)):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                solve_all(FAP_MODE_BATCHED)
                e1.record(stream)
                e1.synchronize()
                p_ms.append(e0.elapsed_time(e1))
            dg.check()
            pm = allmax(float(np.sum(p_ms))) / len(p_ms)
            paths = {"ms_per_step": pm, "pred_ms": pm - ms_per_step,
                     "entries_s": total_entries / (pm * 1e-3),
                     "note": "distances + predecessor rows (int32, same shape) per step"}
            log(f"paths: {pm:.3f} ms/step (+{pm - ms_per_step:.3f} ms for predecessors)")
        except Exception as e:  # noqa: BLE001 - reported, not fatal
            paths = {"unavailable": str(e)[:200]}
            log(f"paths: {e}")
        dg.set_param("paths", 0)

    # ---- plain form ----
    plain_ms = []
    for i in range(1 + args.plain_steps if args.plain_steps > 0 else 0):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solve_all(FAP_MODE_PLAIN)
        e1.record(stream)
        e1.synchronize()
        if i > 0:
            plain_ms.append(e0.elapsed_time(e1))
    dg.check()
    plain_max = allmax(float(np.sum(plain_ms))) if plain_ms else float("nan")
    plain_value = total_entries * len(plain_ms) / (plain_max * 1e-3) if plain_ms else None
    log(f"plain: {plain_ms} ms")

    # ---- roofline figures per stage (algorithmic work of one launch) ----
    m_arcs = int(ro[-1])
    srcs = int(sum(int(bn[p]) for p in mine))
    sssp_bytes = srcs * (4 * (n + 1) + 8 * m_arcs + 4 * n)
    floyd_relax = float(sum(float(vn[p]) ** 3 for p in mine))
    mp_relax = float(sum(float(vn[p] - bn[p]) * float(bn[p]) * n for p in mine))
    mp_bytes = float(sum(4.0 * ((vn[p] - bn[p]) * n + (vn[p] - bn[p]) * bn[p] + bn[p] * n)
                         for p in mine))
    stage_roof = {
        "sssp": {"ms": float(st[0]), "bytes": sssp_bytes,
                 "achieved_gbs": sssp_bytes / (st[0] * 1e-3) / 1e9},
        "gather": {"ms": float(st[1])},
        "floyd": {"ms": float(st[2]), "relax": floyd_relax,
                  "achieved_grelax_s": floyd_relax / (st[2] * 1e-3) / 1e9},
        "minplus": {"ms": float(st[3]), "bytes": mp_bytes, "relax": mp_relax,
                    "achieved_gbs": mp_bytes / (st[3] * 1e-3) / 1e9,
                    "achieved_grelax_s": mp_relax / (st[3] * 1e-3) / 1e9},
    }
    peak_grelax = relax_peak / 1e9
    dom = max(("sssp", "floyd", "minplus"), key=lambda k: stage_roof[k]["ms"])
    if dom == "floyd":
        a = stage_roof["floyd"]["achieved_grelax_s"]
        roof = {"kernel": "floyd_part_kernel", "bound": "dpx", "achieved": a,
                "peak": peak_grelax, "unit": "Grelax/s", "frac": a / peak_grelax,
                "peak_source": "measured relaxation microbenchmark (fap_measure_relax_peak)",
                "traffic": read_traffic(wl.name, "floyd_part_kernel")}
    else:
        thin_only = all(int(bn[p]) <= 16 for p in mine)
        kern = (("msbf_iter_kernel" if "Bellman-Ford" in stage1_used else "sssp_frontier_kernel")
                if dom == "sssp" else
                "minplus_thin_kernel" if thin_only else "minplus_part_kernel")
        a = stage_roof[dom]["achieved_gbs"]
        roof = {"kernel": kern, "bound": "hbm", "achieved": a, "peak": hbm_peak, "unit": "GB/s",
                "frac": a / hbm_peak, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": read_traffic(wl.name, kern)}
    stage_roof["floyd"]["frac_of_relax_peak"] = stage_roof["floyd"]["achieved_grelax_s"] / peak_grelax
    stage_roof["minplus"]["frac_of_relax_peak"] = (stage_roof["minplus"]["achieved_grelax_s"]
                                                   / peak_grelax)
    stage_roof["minplus"]["frac_of_hbm"] = stage_roof["minplus"]["achieved_gbs"] / hbm_peak
    form_now = (solve_tuned["params"] if solve_tuned else
                {"minplus_pack16": int(not args.no_pack16), "floyd_queue": int(not args.no_queue)})
    if (form_now["floyd_queue"] and stage1_used.startswith("SSSP")
            and (dtype != 0 or not form_now["minplus_pack16"])):
        stage_roof["minplus"]["note"] = ("the min-plus tiles of parts with more than 16 boundary vertices "
                                         "ran inside the Floyd work queue: their time is in the floyd stage")
    stage_roof["sssp"]["frac_of_hbm"] = stage_roof["sssp"]["achieved_gbs"] / hbm_peak

    # ---- e2e through the public API: host inputs in, every block out ----
    del dg
    torch.cuda.synchronize()
    if args.e2e_steps > 0 and world == 1 and len(groups) > 1:
        log("e2e with grouped output")
    max_rows = int(max(vn[p] for p in mine))
    # two pinned host buffers: each block's copy is queued on one of the
    # library's two copy slots, so that the next block's conversion to
    # float32 overlaps this block's device-to-host copy
    host_bufs = [torch.empty((max_rows, n), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    hbs = [b.numpy() for b in host_bufs]
    pin = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy()
           for k, v in dict(ro=ro, col=col, w=w.astype(np.float32), gid=gid, st2ed=st2ed,
                            vn=vn, vo=vo, bn=bn).items()}
    h2d = sum(a.nbytes for a in pin.values())
    d2h = my_rows * n * 4
    e2e_s = []
    for i in range(1 + args.e2e_steps if args.e2e_steps > 0 else 0):
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        g2 = DeviceGraph(ctx, pin["ro"], pin["col"], pin["w"])
        g2.set_parts(wl.K, pin["gid"], pin["st2ed"], pin["vn"], pin["vo"], pin["bn"])
        g2.reserve(max(rows_of(g, vn) for g in groups))
        if staged:
            g2.cache_build()
        if shard is not None:
            owner_, stride_, send_, recv_ = shard
            g2.shard_begin(mine, send_.data_ptr(), stride_)
            dist.all_gather_into_tensor(recv_, send_)
            g2.shard_finish(recv_.data_ptr(), world, owner_, stride_)
        k = 0
        for grp in groups:
            g2.solve(grp, FAP_MODE_BATCHED)
            for p in grp:
                g2.copy_block_async(p, hbs[k % 2][:int(vn[p])], k % 2, out_dtype=FAP_DTYPE_F32)
                k += 1
            for slot in range(2):   # the group's blocks are out before its rows are reused
                g2.copy_wait(slot)
        t1 = time.perf_counter()
        del g2
        if i > 0:
            e2e_s.append(t1 - t0)
    e2e_max = allmax(float(np.sum(e2e_s)))
    e2e_value = total_entries * len(e2e_s) / e2e_max if e2e_s else None
    log(f"e2e: {e2e_s} s/step")

    # ---- serving stream (rank 0, N=1 only) ----
    serving = None
    if rank == 0 and world == 1 and not args.no_serve:
        del host_bufs, hbs
        torch.cuda.empty_cache()
        serving = run_serving(args, local)

    # ---- further workloads (rank 0, N=1 only); their reference parity
    # processes started before the headline measurement ----
    extras = None
    if extra_jobs:
        extras = {}
        torch.cuda.empty_cache()
        for name, job in extra_jobs.items():
            gpu = None
            try:
                if isinstance(job, Exception):
                    raise job
                extras[name], gpu, xdtype = run_extra(args, job, ctx, relax_peak, hbm_peak, peak_kind)
                extras[name]["parity"] = finish_extra_parity(job, gpu, xdtype)
                log(f"{name}: parity {extras[name]['parity']}")
            except Exception as e:  # noqa: BLE001 - reported in the line, not fatal
                extras[name] = {"unavailable": str(e)[:300]}
                log(f"{name}: {e}")
            del gpu
            torch.cuda.empty_cache()

    # ---- CPU baseline (rank 0, N=1 only) and parity of the same parts ----
    cpu = None
    parity = None
    if cpu_leg:
        from oracle import oracle as O
        P = cpu_procs(args.cpu_procs)
        parts = parity_parts
        with tempfile.TemporaryDirectory() as tmp:
            # the GPU run's partition (0-based part ids), so that both solve
            # the same parts; process 0 also dumps the reference's renumbering
            pfile = os.path.join(tmp, "partition.bin")
            (np.asarray(gid, dtype=np.int64) - 1).astype(np.int32).tofile(pfile)
            meta_f = os.path.join(tmp, "meta.bin")
            extra, files = {0: ["--meta", meta_f]}, {}
            for i, p in enumerate(parts):
                if dtype == 0:
                    files[p] = os.path.join(tmp, f"rowsum_{p}.bin")
                    extra.setdefault(i, []).extend(["--rowsum", files[p]])
                elif i < PARITY_FLOAT_PARTS:
                    files[p] = os.path.join(tmp, f"dist_{p}.bin")
                    extra.setdefault(i, []).extend(["--dist", files[p]])
            kind, res = run_reference_sample(wl, [[p] for p in parts], P, extra=extra,
                                             partition_file=pfile)
            if kind == "reference":
                parity = compare_parity(wl, gpu_par, files, dtype, st2ed, O.read_meta(meta_f))
            else:
                parity = {"unavailable": "reference binary absent (C restatement timed instead)"}
        del gpu_par
        ent = sum(r[0][2] for r in res)
        sec = max(r[0][3] for r in res)
        cpu = {"value": ent / sec, "unit": UNIT, "cores": P, "kind": kind,
               "sample": f"{P} parts of {wl.name} (K={wl.K}), one process per core, "
                         f"1 thread each; time = slowest process ({sec:.2f} s)"}
        log(f"parity vs reference on {len(files)} sampled parts: {parity}")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "int32" if dtype == 0 else "f32",
            "data": wl.data_description(),
            "config": common_config(wl.describe(), world),
            "solve": {"mode": "batched", "stage1": stage1_used,
                      "groups": len(groups),
                      "stage_cache": ({"note": "stages 1-2 of every part once per step (resident cache), "
                                               "then each group's min-plus merge",
                                       "phases_ms": np.round(np.mean(cache_phases, 0), 3).tolist(),
                                       "phases": ("local closures, boundary-graph closure, expansion, fix-up"
                                                  if "boundary graph" in stage1_used else
                                                  "SSSP, gather, Floyd, -")}
                                      if staged and cache_phases else None),
                      "sssp_delta": {"value": tuned["delta"], "factor_of_mean_weight": tuned["factor"],
                                     "bucket": tuned["key"], "from_cache": tuned["cached"]},
                      "solve_form": ({"params": solve_tuned["params"], "candidates_ms": solve_tuned["ms"],
                                      "from_cache": solve_tuned["cached"]} if solve_tuned else
                                     {"params": {"minplus_pack16": int(not args.no_pack16),
                                                 "floyd_queue": int(not args.no_queue)}})},
            "plain": {"value": plain_value, "ms_per_step": plain_max / max(len(plain_ms), 1),
                      "steps": len(plain_ms)},
            "batched_over_plain": (value / plain_value) if plain_value else None,
            "stages_ms": {"sssp": float(st[0]), "gather": float(st[1]), "floyd": float(st[2]),
                          "minplus": float(st[3]), "total": float(st[4])},
            "roofline": roof, "stage_roofline": stage_roof,
            "relax_peak_grelax_s": peak_grelax,
            "cpu_baseline": cpu,
            "parity": parity,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": len(e2e_s),
                    "s_per_step": e2e_max / max(len(e2e_s), 1)},
            "gpu_launches": int(launches),
            "clocks": clk,
            "serving": serving,
            "paths": paths,
            "workloads": extras,
        }
        emit(line)
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse_args()
    if args.impl == "reference":
        main_reference(args)
    else:
        main_fap(args)


if __name__ == "__main__":
    main()
