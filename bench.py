"""Benchmark: FK-PK hash join + aggregation on one B200 (or N replicas).

Workload (the configuration the headline metric is quoted on): a 1,500,000-row
dimension with unique int32 keys filtered on ``segment == 1`` (20%) and built
into a hash table, probed by a 6,000,000-row fact table (int32 FK + int64
measure), grouped by ``nation`` (25 groups) with an exact 64-bit sum and a count.
Seeded synthetic data with those shapes (no TPC-H data here).

A step is one execution of the whole plan (dimension build pipeline, fact probe
+ aggregate pipeline, aggregation output pipeline).  ``value`` counts the input
rows of both tables per second of device time (CUDA events on the engine's
stream), inputs resident in HBM; the inputs (90 MB) fit in L2, so between steps
a 256 MB buffer is written and another 256 MB read (the read writes the dirty
flush lines back before the timed region).  ``e2e`` runs the same plan through
the public API with the input columns copied from pinned host memory every step
and the result read back, timed on the host.  ``roofline`` is for the dominant
kernel (the slowest pipeline: the fact probe), its algorithmic bytes the columns
it reads; ``traffic`` is its DRAM bytes from the committed ncu summary
(profiles/traffic.json).  ``--impl reference`` times the CPU oracle (numpy
restatement of the reference's semantics), partitioned over all host cores.

``--workload c0|c2|c3`` measures the other configurations the same way (scan-
filter-aggregate, divergent multimap expansion, three-way star join) for the
per-pipeline table; the headline line is the default ``c1``.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from dogqc_b200 import replicas  # noqa: E402  (after the path insert)

SCALE = 1.0
WORKLOAD = "c1"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
METRIC = "rows/s (FK-PK hash join + aggregate pipeline, input rows of both tables per second)"
CONFIG = {"workload": "fk_pk_join_agg", "dim_rows": 1_500_000, "fact_rows": 6_000_000,
          "dim_filter": "segment == 1 (20%)", "groups": 25, "l2": "256 MB write + 256 MB read between steps (inputs evicted)",
          "parallelism": "replicas"}
# the other configurations (parity-test cases; measured with --workload for the
# per-pipeline roofline table)
WORKLOADS = {
    "c0": ("rows/s (scan-filter-aggregate pipeline, input rows per second)",
           {"workload": "scan_filter_agg", "rows": 6_000_000, "filter": "shipdate <= max-90",
            "groups": 6, "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c1": (METRIC, CONFIG),
    "c2": ("rows/s (multimap build + divergent expansion, input rows of both tables per second)",
           {"workload": "divergent_expansion", "build_rows": 10_000_000, "probe_rows": 16_777_216,
            "build_keys": "zipf(1.0) over 100,000", "probe_keys": "uniform over 200,000",
            "filters": "90/50/10/1%", "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c3": ("rows/s (three-way star join + 1M-group aggregate, input rows per second)",
           {"workload": "star_join_high_cardinality", "fact_rows": 60_000_000,
            "dim_rows": [1_500_000, 200_000, 10_000], "groups": "~1,000,000",
            "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c7": ("rows/s (one-row aggregate nested-loop joined to every row + group by, input rows per second)",
           {"workload": "nested_loop_join_scalar_subquery", "customer_rows": 150_000,
            "condition": "acctbal > avg(acctbal)", "groups": 25,
            "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c8": ("rows/s (temp table written by one plan root, scanned and joined by another, input rows per second)",
           {"workload": "temp_table_two_roots", "customer_rows": 150_000, "order_rows": 1_500_000,
            "orders_filter": "flag < 50 (50%)", "customers_filter": "nation < 5 (20%)",
            "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c9": ("rows/s (filter + group by two variable-length strings, string result columns, input rows per second)",
           {"workload": "string_group_by", "rows": 6_000_000, "filter": "receiptdate < middle (50%)",
            "groups": 28, "keys": "ship mode, ship instruction (variable-length strings)",
            "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c10": ("rows/s (FK-PK join carrying a string from the build side + group by it, input rows of both tables per second)",
            {"workload": "join_string_payload_group_by", "customer_rows": 150_000, "order_rows": 1_500_000,
             "groups": 5, "key": "market segment (a string of the build side)",
             "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c5": ("rows/s (left outer join on a multimap + two aggregations, input rows of both tables per second)",
           {"workload": "outer_join_two_aggregations", "customer_rows": 150_000, "order_rows": 1_500_000,
            "orders_filter": "flag >= 2 (98%)", "customers_without_orders": "1/3",
            "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c11": ("rows/s (EXISTS on a unique key filter table + group by, input rows of both tables per second)",
            {"workload": "semi_join_exists", "order_rows": 1_500_000, "lineitem_rows": 6_000_000,
             "orders_filter": "one quarter (3.6%)", "lineitem_filter": "commit < receipt (~48%)", "groups": 5,
             "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c12": ("rows/s (EXISTS and NOT EXISTS with <> conditions walked over multimaps, input rows per second)",
            {"workload": "semi_anti_join_conditions", "order_rows": 1_500_000, "lineitem_rows": "3 x 6,000,000",
             "groups": "~10,000",
             "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c13": ("rows/s (NOT EXISTS on a unique key filter table + group by, input rows of both tables per second)",
            {"workload": "anti_join_not_exists", "customer_rows": 150_000, "order_rows": 1_500_000, "groups": 25,
             "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c14": ("rows/s (TPC-H Q16 shape: string predicates, FK-PK join, anti join, two aggregations with string keys, "
            "input rows of the tables read per second)",
            {"workload": "q16_strings", "part_rows": 200_000, "partsupp_rows": 800_000, "supplier_rows": 10_000,
             "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c15": ("rows/s (FK-PK join on a string key + group by, input rows of both tables per second)",
            {"workload": "string_key_join", "nation_rows": 25, "supplier_rows": 100_000,
             "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c16": ("rows/s (TPC-H Q22 shape: substrings in an IN list and as a group key, nested-loop join with an "
            "average, NOT EXISTS, input rows of the tables read per second)",
            {"workload": "q22_substrings", "customer_rows": "2 x 150,000", "order_rows": 1_500_000,
             "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c17": ("rows/s (TPC-H Q13 shape: NOT LIKE on comments, outer join, two aggregations, input rows per second)",
            {"workload": "q13_comments", "customer_rows": 150_000, "order_rows": 1_500_000,
             "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c18": ("rows/s (TPC-H Q20 shape: LIKE prefix, aggregation into a two-key join table, semi joins, string "
            "results, input rows of the tables read per second)",
            {"workload": "q20_strings", "lineitem_rows": 6_000_000, "partsupp_rows": 800_000, "part_rows": 200_000,
             "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
    "c19": ("rows/s (TPC-H Q2 shape: LIKE suffix, MIN joined back, string results, input rows of the tables read "
            "per second)",
            {"workload": "q2_strings", "partsupp_rows": "2 x 800,000", "part_rows": "2 x 200,000",
             "supplier_rows": "2 x 10,000",
             "l2": "256 MB write + 256 MB read between steps (inputs evicted)", "parallelism": "replicas"}),
}


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def load_profile_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(WORKLOAD, {}).get("dram_bytes_per_launch")
    except Exception:
        return None


def pipeline_bytes(db, lowering, i):
    """Algorithmic bytes of pipeline i: every column it reads, once, at stored width."""
    pipe = lowering.pipes[i]
    if not pipe.table:
        return 0
    from dogqc_b200.database import StringColumn
    table = db[pipe.table]
    total = 0
    for c in pipe.cols:
        col = table.columns[c]
        if isinstance(col, StringColumn):  # fixed-width strings are read without offsets
            total += col.chars.nbytes + (0 if col.width else col.offsets.nbytes)
        else:
            total += col.nbytes
    return total


def join_pairs(db):
    """Matching (probe, build) key pairs of the divergent-expansion workload."""
    import numpy as np
    b = np.bincount(db["r_build"].columns["r_key"])
    p = np.bincount(db["s_probe"].columns["s_key"])
    n = min(len(b), len(p))
    return int((b[:n].astype(np.int64) * p[:n].astype(np.int64)).sum())


class ClockSampler(object):
    """SM clock and clock-event (throttle) reasons sampled through NVML every few
    milliseconds while the timed region runs (the counters nvidia-smi reports as
    clocks.sm and clocks_event_reasons.*)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, device, period=0.002):
        self.device = device
        self.period = period
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self.nvml = None
        self.stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.nvml = pynvml
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        except Exception:
            self.nvml = None
        return self

    def _run(self):
        nv = self.nvml
        while not self.stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for name, mask in self.REASONS.items():
                    if bits & mask:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(self.period)

    def __exit__(self, *exc):
        self.stop.set()
        if self.nvml:
            self.thread.join(timeout=2)

    def summary(self):
        mhz = sorted(self.samples)
        return {"sm_mhz": mhz[len(mhz) // 2] if mhz else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(mhz), "source": "nvml"}


def dist_setup():
    return replicas.setup()


def dist_max(x, world):
    return replicas.max_over_ranks(x, world)


def dist_barrier(world):
    replicas.barrier(world)


def build_plan(db):
    from dogqc_b200 import workloads
    from dogqc_b200.relational import RelationalAlgebra
    alg = RelationalAlgebra(db)
    plan, cfg = workloads.build(WORKLOAD, alg, scale=SCALE)
    return alg.resolveAlgebraPlan(plan, cfg)


# ------------------------------------------------------------------ our arm --

def input_rows(db):
    """Rows of the tables the workload's plan scans (a table it does not read is
    not counted)."""
    from dogqc_b200.lowering import Lowering
    read = {p.table for p in Lowering(build_plan(db)).pipes if p.table}
    return sum(t.size for name, t in db.tables.items() if name in read)


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    from dogqc_b200 import workloads
    from dogqc_b200.engine import Engine

    torch.cuda.set_device(local)
    db = workloads.GENERATORS[WORKLOAD](SCALE)
    plan = build_plan(db)
    rows_per_step = input_rows(db)
    engine = Engine(local, tile_rows=args.tile_rows, ctas_per_sm=args.ctas_per_sm, flags=args.engine_flags)
    engine.register_database(db)
    # L2 flush between steps: write 256 MB (evicts the inputs), then read another
    # 256 MB, which writes the dirty flush lines back before the timed region
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    evict = torch.zeros(32 << 20, dtype=torch.int64, device="cuda")

    def flush_l2():
        flush.fill_(1)
        evict.sum()

    # the plan's launch shapes and table sizing, picked by measurement on this
    # GPU (each candidate run after an L2 flush) before anything is timed
    tuning, tuned = None, None
    if args.tuning:
        tuning = json.loads(args.tuning)
        tuned = {"tuning": tuning, "given": True}
    elif not args.no_autotune:
        from dogqc_b200 import autotune
        from dogqc_b200.lowering import Lowering
        t0 = time.perf_counter()
        tuning, t_best, log = autotune.tune_plan(engine, Lowering(plan), reps=5, between=flush_l2)
        tuned = {"tuning": tuning, "candidates": len(log), "best_ms": t_best * 1e3 if t_best else None,
                 "search_s": round(time.perf_counter() - t0, 1)}
    p = engine.prepare(plan, tuning=tuning)
    npipes = len(p.lowering.pipes)

    def timed(plan_, steps):
        """Warm-up, then `steps` executions each after an L2 flush: summed
        device time of the runs (CUDA events on the engine's stream), summed
        per-pipeline times (zero where the run replayed a graph), launches."""
        def step():
            flush_l2()
            torch.cuda.synchronize()
            res_ = plan_.execute()
            return res_, plan_.timing()
        for _ in range(args.warmup):
            res_, _ = step()
        dist_barrier(world)
        torch.cuda.synchronize()
        tot, launches_ = 0.0, 0
        pipes = [0.0] * len(plan_.lowering.pipes)
        for _ in range(steps):
            res_, t = step()
            tot += t["total_ms"]
            for i in range(len(pipes)):
                pipes[i] += t["pipeline_ms"][i]
            launches_ += t["kernel_launches"]
        torch.cuda.synchronize()
        dist_barrier(world)
        return res_, dist_max(tot, world), [dist_max(x, world) for x in pipes], launches_

    # the plan as dq_plan_execute runs it: after the first run, its launches
    # replay from a captured CUDA graph
    with ClockSampler(local) as clocks:
        res, total_ms, _, launches = timed(p, args.steps)
    # per-kernel times need events between the launches: the same plan on a
    # second context that does not capture graphs, over as many steps
    kengine = Engine(local, tile_rows=args.tile_rows, ctas_per_sm=args.ctas_per_sm, flags=args.engine_flags | 2)
    kengine.register_database(db)
    kp = kengine.prepare(plan, tuning=tuning)
    _, k_total_ms, pipe_ms, _ = timed(kp, args.steps)
    kp.free()
    dom = max(range(npipes), key=lambda i: pipe_ms[i])   # the dominant pipeline kernel
    probe_ms = pipe_ms[dom]
    # the same launch's streaming bound: one generated kernel that reads the
    # dominant pipeline's columns (same table, same bytes) and only sums them
    stream_ms = None
    dp = p.lowering.pipes[dom]
    if dp.table and not args.no_stream_bound:
        from dogqc_b200.database import StringColumn
        from dogqc_b200.relational import RelationalAlgebra, Reduction
        cols = [c for c in dp.cols if not isinstance(db.tables[dp.table].columns[c], StringColumn)]
        if cols:
            salg = RelationalAlgebra(db)
            sagg = salg.aggregation([], [(Reduction.SUM, c, "sum_%d" % i) for i, c in enumerate(cols)], salg.scan(dp.table))
            sp = kengine.prepare(salg.resolveAlgebraPlan(sagg, {}))
            _, _, s_pipe_ms, _ = timed(sp, args.steps)
            sp.free()
            stream_ms = s_pipe_ms[0] / args.steps
    kengine.close()
    fact_bytes = pipeline_bytes(db, p.lowering, dom)
    ms_per_step = total_ms / args.steps
    value = rows_per_step * world / (ms_per_step / 1e3)

    # end to end: host columns (pinned) -> device, execute, result back.  String
    # columns (a dimension's text) stay resident: the library does not update
    # them in place, and they are not counted in the copied bytes.
    from dogqc_b200.database import StringColumn
    d2h_rows = res.nrows
    d2h = sum(c.nbytes for c in res.columns) + 12
    e2e_value = None
    h2d = 0
    if not args.no_e2e:
        pinned = {}
        read = {pp.table for pp in p.lowering.pipes if pp.table}
        for tname, table in db.tables.items():
            if tname not in read:
                continue
            for cname, col in table.columns.items():
                if isinstance(col, StringColumn):
                    continue
                arr = np.ascontiguousarray(col)
                t = torch.from_numpy(arr.view(np.uint8)).pin_memory()
                pinned[(tname, cname)] = (t, arr.dtype)

        class PinnedTable(object):
            def __init__(self, table):
                self.name = table.name
                self.size = table.size
                self.types = table.types
                self.columns = {c: pinned[(table.name, c)][0].numpy().view(pinned[(table.name, c)][1])
                                for c in table.columns if (table.name, c) in pinned}

        ptables = [PinnedTable(t) for t in db.tables.values() if t.name in read]
        h2d = sum(t.nbytes for t, _ in pinned.values())
        for _ in range(2):
            for pt in ptables:
                engine.update_table(pt)
            p.execute()
        dist_barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            for pt in ptables:
                engine.update_table(pt)
            r2 = p.execute()
        e2e_s = time.perf_counter() - t0
        e2e_s = dist_max(e2e_s, world)
        assert r2.nrows == d2h_rows
        e2e_value = rows_per_step * world * args.steps / e2e_s

    peak, peak_kind = hbm_peak()
    probe_avg_s = probe_ms / args.steps / 1e3
    achieved = fact_bytes / probe_avg_s / 1e9
    plan_bytes = sum(pipeline_bytes(db, p.lowering, i) for i in range(npipes))
    metric, config = WORKLOADS[WORKLOAD]
    kernel = "dq_main (generated kernel of pipeline %d: %s)" % (dom, p.lowering.pipes[dom].table or "scan of a temp table")
    if args.engine_flags & 12:
        kernel = "prebuilt %s kernel of pipeline %d" % ("row" if args.engine_flags & 4 else "tile", dom)
    out = {
        "metric": metric, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)",
        "config": config,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": load_profile_traffic(),
                     "kernel": kernel,
                     "algorithmic_bytes": fact_bytes, "avg_ms": probe_avg_s * 1e3,
                     "peak_source": "%s hbm_gbs (burst copy)" % peak_kind,
                     "stream_ms": stream_ms,
                     "frac_of_stream": stream_ms / (probe_avg_s * 1e3) if stream_ms else None,
                     "stream_source": "one generated kernel summing the same columns of the same table "
                                      "(the kernel's reads without its probes, groups or refill)"},
        "plan": {"algorithmic_bytes": plan_bytes, "avg_ms": ms_per_step,
                 "frac": plan_bytes / (ms_per_step / 1e3) / 1e9 / peak,
                 "replayed_graph": True,
                 "no_graph_avg_ms": k_total_ms / args.steps,
                 "pipeline_ms": [x / args.steps for x in pipe_ms],
                 "pipeline_ms_source": "second timed loop without graph replay (events between launches)"},
        "e2e": {"value": e2e_value, "unit": "rows/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "autotune": tuned,
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    if WORKLOAD == "c2":
        pairs = join_pairs(db)
        out["join_pairs"] = {"pairs": pairs, "pairs_per_s": pairs * world / (ms_per_step / 1e3)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(db, plan)
        out["ref_gpu_baseline"] = ref_gpu_baseline(db)
    engine.close()
    return out


# ------------------------------------------------------------ CPU baselines --

def _cpu_eval():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_eval
    return cpu_eval


def _sized_for(db, plan, seconds, runs):
    """The workload, or a smaller seeded instance of the same shape, such that
    `runs` evaluations on all cores take about `seconds` (one run is timed
    first, after a warm-up run)."""
    from dogqc_b200 import workloads
    cpu = _cpu_eval()
    prep = cpu.Prepared(db, plan)
    prep.run()                       # warm-up: first touches of fresh memory
    one = prep.run()[2]
    scale, what = SCALE, "the full workload"
    if one * runs > seconds:
        scale = SCALE * seconds / (one * runs)
        db = workloads.GENERATORS[WORKLOAD](scale)
        plan = build_plan(db)
        prep = cpu.Prepared(db, plan)
        prep.run()
        what = "the same workload at scale %.4f" % scale
    return db, plan, prep, what


def cpu_baseline(db, plan, seconds=15.0, repeats=5):
    """The multithreaded C++ evaluation of the same plan IR (oracle/cpu_eval.cpp)
    on all host cores: the median of `repeats` warm runs, on the full workload
    or, above about `seconds` of CPU time, a smaller seeded instance of it."""
    cpu = _cpu_eval()
    db, plan, prep, what = _sized_for(db, plan, seconds, repeats)
    times = sorted(prep.run()[2] for _ in range(repeats))
    dt = times[len(times) // 2]
    rows = input_rows(db)
    return {"value": rows / dt, "unit": "rows/s", "cores": prep.threads, "kind": "port",
            "sample": "median of %d warm runs of %s (%d input rows) through the C++ evaluator of the plan IR "
                      "(oracle/cpu_eval.cpp), %d threads" % (repeats, what, rows, prep.threads),
            "ms_per_run": dt * 1e3}


def ref_gpu_baseline(db, runs=5):
    """The reference's own generated pipeline for this workload (its CUDA
    source from its translator, compiled for sm_100a into oracle/_ref/bin by
    oracle/ref_harness.py) run on the same seeded tables in this bench run:
    medians of its own <timing> block (std::clock around each synchronised
    launch) over `runs` runs."""
    import shutil
    import subprocess
    import tempfile
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from mmdb import write_mmdb
    from ref_run import parse_timing
    exe = os.path.join(ROOT, "oracle", "_ref", "bin", WORKLOAD)
    if SCALE != 1.0 or not os.path.exists(exe):
        return {"unavailable": "no reference binary for %s at scale %g" % (WORKLOAD, SCALE)}
    work = tempfile.mkdtemp(prefix="dq_refgpu_")
    try:
        write_mmdb(db, os.path.join(work, "mmdb"))
        timings = []
        for _ in range(runs):
            p = subprocess.run([exe], cwd=work, capture_output=True, timeout=300)
            if p.returncode != 0:
                return {"unavailable": "reference binary exited with %d" % p.returncode}
            timings.append(parse_timing(p.stdout.decode("latin-1")))
    finally:
        shutil.rmtree(work, ignore_errors=True)
    med = {}
    for k in timings[0]:
        vals = sorted(t.get(k, 0.0) for t in timings)
        med[k] = vals[len(vals) // 2]
    total = med.get("totalKernelTime", 0.0)
    rows = input_rows(db)
    return {"binary": "oracle/_ref/bin/%s (the reference's generated pipeline, sm_100a)" % WORKLOAD,
            "runs": runs, "kernel_ms": {k: v for k, v in med.items() if k.startswith("krnl_")},
            "total_kernel_ms": total, "rows_per_s": rows / (total / 1e3) if total else None,
            "timer": "the program's own <timing>: std::clock around each launch and its synchronisation, "
                     "0.1 ms resolution"}


def run_reference(args, world, rank):
    """The CPU reference arm: the C++ evaluator of the same plan IR on all host
    cores, one evaluation per step (of a smaller seeded instance of the same
    workload when `steps` full evaluations would take more than two minutes)."""
    if rank != 0:
        return None
    from dogqc_b200 import workloads
    db = workloads.GENERATORS[WORKLOAD](SCALE)
    plan = build_plan(db)
    db, plan, prep, what = _sized_for(db, plan, 120.0, args.warmup + args.steps)
    rows = input_rows(db)
    times = []
    for i in range(args.warmup + args.steps):
        dt = prep.run()[2]
        if i >= args.warmup:
            times.append(dt)
    step_s = sum(times) / len(times)
    value = rows / step_s
    metric, config = WORKLOADS[WORKLOAD]
    return {
        "metric": metric, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)",
        "config": config, "impl": "reference",
        "cpu_baseline": {"kind": "port", "cores": prep.threads, "value": value, "unit": "rows/s",
                         "sample": "one evaluation of %s (%d input rows) per step through the C++ evaluator "
                                   "of the plan IR (oracle/cpu_eval.cpp), %d threads" % (what, rows, prep.threads)},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------- batched and served forms --

def run_batched(args, world, rank, local):
    """256 divergent-expansion instances (row counts log-uniform in 2^10..2^20)
    in one batch (one generated kernel per pipeline, one CUDA graph) against the
    same instances executed as plain plans one after the other."""
    import numpy as np
    import torch
    from dogqc_b200 import autotune, batch
    from dogqc_b200.engine import Engine
    torch.cuda.set_device(local)
    n = 256
    insts = batch.make_instances("c2", n)
    rows = sum(i.input_rows for i in insts)
    engine = Engine(local)
    batch.register(engine, insts)
    tuning, tuned = None, None
    if args.autotune:
        tuning, t_best, log = autotune.tune_batch(engine, [i.lowering for i in insts])
        tuned = {"tuning": tuning, "candidates": len(log), "best_ms": t_best * 1e3}
    b = batch.prepare_batch(engine, insts, tuning)
    for _ in range(args.warmup):
        res = b.execute()
    dist_barrier(world)
    ms = []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            b.execute()
            ms.append(b.timing()["total_ms"])
    step_ms = dist_max(float(np.mean(ms)), world)
    from dogqc_b200 import serve
    plans = batch.prepare_one_by_one(engine, insts)
    order = [(0.0, i) for i in range(n)]
    keyed = {i: p for i, p in enumerate(plans)}
    serve.sequence(engine, insts, order, keyed)
    seq = []
    for _ in range(max(1, args.steps // 4)):
        per, wall, _ = serve.sequence(engine, insts, order, keyed)
        seq.append(wall)
    one_ms = float(np.median(seq)) * 1e3
    parity = all(sorted(p.execute().rows()) == sorted(r.rows()) for p, r in zip(plans, res))
    out = {
        "metric": "instances/s (256 divergent-expansion instances, one batch)", "value": n * world / (step_ms / 1e3),
        "unit": "instances/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded)",
        "config": {"workload": "divergent_expansion_x256", "instances": n, "rows": "log-uniform 2^10..2^20 probe rows",
                   "input_rows": rows, "parallelism": "replicas"},
        "rows_per_s": rows * world / (step_ms / 1e3),
        "one_by_one": {"ms": one_ms, "instances_per_s": n / (one_ms / 1e3),
                       "how": "the same instances as plain plans, executed one after the other from native code"},
        "speedup_vs_one_by_one": one_ms / step_ms,
        "parity_with_one_by_one": parity,
        "gpu_launches": b.timing()["kernel_launches"] * args.steps,
        "clocks": clocks.summary(),
    }
    if tuned:
        out["autotune"] = tuned
    b.free()
    for p in plans:
        p.free()
    engine.close()
    return out


TBL_BLOCK = 100_000
TBL_WORDS = [b"carefully", b"final", b"deposits", b"furiously", b"regular", b"accounts", b"blithely",
             b"ironic", b"packages", b"quickly", b"express", b"pending", b"requests", b"slyly", b"bold"]
def tbl_fields():
    from dogqc_b200 import _lib as L
    dec = lambda n: (n, L.TEXT_DECIMAL, 2)  # noqa: E731
    return [("l_orderkey", L.TEXT_INT), ("l_partkey", L.TEXT_INT), ("l_suppkey", L.TEXT_INT),
            ("l_linenumber", L.TEXT_INT), ("l_quantity", L.TEXT_INT), dec("l_extendedprice"), dec("l_discount"),
            dec("l_tax"), ("l_returnflag", L.TEXT_CHAR), ("l_linestatus", L.TEXT_CHAR),
            ("l_shipdate", L.TEXT_DATE), ("l_commitdate", L.TEXT_DATE), ("l_receiptdate", L.TEXT_DATE),
            ("l_shipinstruct", L.TEXT_STRING), ("l_shipmode", L.TEXT_STRING), ("l_comment", L.TEXT_STRING)]


def tbl_text(rows, seed=20261203):
    """lineitem as dbgen writes it (16 fields, each followed by '|', the types of
    the reference's schema, query/schema/tpch.py:22-41): a block of
    100,000 seeded lines repeated to ``rows`` lines.  Returns the text and the
    expected sums of l_orderkey and l_extendedprice (cents)."""
    import numpy as np
    r = np.random.Generator(np.random.Philox(seed))
    n = min(rows, TBL_BLOCK)
    ok = r.integers(1, 6_000_000, n)
    pk = r.integers(1, 200_000, n)
    sk = r.integers(1, 10_000, n)
    ln = r.integers(1, 8, n)
    qty = r.integers(1, 51, n)
    price = r.integers(90_000, 10_500_001, n)
    disc = r.integers(0, 11, n)
    tax = r.integers(0, 9, n)
    rf = r.integers(0, 3, n)
    ls = r.integers(0, 2, n)
    day = r.integers(0, 2526, n)
    nw = r.integers(2, 8, n)
    words = r.integers(0, len(TBL_WORDS), (n, 8))
    instr = [b"DELIVER IN PERSON", b"COLLECT COD", b"NONE", b"TAKE BACK RETURN"]
    modes = [b"TRUCK", b"MAIL", b"REG AIR", b"AIR", b"FOB", b"RAIL", b"SHIP"]
    im = r.integers(0, 4, n)
    mm = r.integers(0, 7, n)

    def date(d):
        y, rem = 1992 + d // 365, d % 365
        return b"%04d-%02d-%02d" % (y, rem // 28 % 12 + 1, rem % 28 + 1)
    lines = []
    for i in range(n):
        d = int(day[i])
        lines.append(b"%d|%d|%d|%d|%d|%d.%02d|0.%02d|0.%02d|%c|%c|%s|%s|%s|%s|%s|%s|\n" % (
            ok[i], pk[i], sk[i], ln[i], qty[i], price[i] // 100, price[i] % 100, disc[i], tax[i],
            b"ANR"[rf[i]], b"FO"[ls[i]], date(d), date(d + 30), date(d + 60), instr[im[i]], modes[mm[i]],
            b" ".join(TBL_WORDS[int(w)] for w in words[i, :nw[i]])))
    block = b"".join(lines)
    reps, rest = divmod(rows, n)
    text = block * reps + b"".join(lines[:rest])
    sum_ok = int(ok.sum()) * reps + int(ok[:rest].sum())
    sum_price = int(price.sum()) * reps + int(price[:rest].sum())
    return text, sum_ok, sum_price


def tbl_algorithmic_bytes(nbytes, rows):
    """Bytes the parse kernel must move: the text, the line ends (8 B a row), the
    fixed-width columns (5 ints, 3 decimals of 8 B, 2 chars, 3 dates) and the
    (first byte, length) record of each of the 3 strings (12 B)."""
    return nbytes + rows * (8 + 5 * 4 + 3 * 8 + 2 * 1 + 3 * 4 + 3 * 12)


TBL_REF_ROWS = 2_000_000


def tbl_cpu_baseline(fields):
    """The reference's own importer (generated C++, compiled here by
    oracle/build_ref_importer.py into oracle/_ref) on the first 2,000,000 lines
    of the benchmark text, timed on the host; without that program, the Python
    restatement of it on the first 3 MB."""
    import shutil
    import tempfile
    refbin = os.path.join(ROOT, "oracle", "_ref", "tbl_import_lineitem_%d" % TBL_REF_ROWS)
    if os.path.exists(refbin):
        sample = tbl_text(TBL_REF_ROWS)[0]
        work = tempfile.mkdtemp(prefix="dq_tbl_ref_")
        try:
            os.makedirs(os.path.join(work, "csv"))
            os.makedirs(os.path.join(work, "mmdb"))
            with open(os.path.join(work, "csv", "lineitem.tbl"), "wb") as fh:
                fh.write(sample)
            t0 = time.perf_counter()
            subprocess.run([refbin], cwd=work, check=True, stdout=subprocess.DEVNULL)
            dt = time.perf_counter() - t0
        finally:
            shutil.rmtree(work, ignore_errors=True)
        return {"value": len(sample) / dt / 1e9, "unit": "GB/s", "cores": 1, "kind": "reference",
                "sample": "the first %d lines (%d bytes) of the same text through the reference's generated "
                          "importer (its CSV reader, both passes, column files written), wall time" % (
                              TBL_REF_ROWS, len(sample)), "seconds": dt}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import text_import
    text = tbl_text(30_000)[0]
    t0 = time.perf_counter()
    text_import.parse(text, [(f[0], f[1]) + tuple(f[2:]) for f in fields])
    dt = time.perf_counter() - t0
    return {"value": len(text) / dt / 1e9, "unit": "GB/s", "cores": 1, "kind": "port",
            "sample": "30,000 lines (%d bytes) through the Python restatement of the reference's importer" % len(text)}


def run_import(args, world, rank, local):
    """Text import: lineitem in dbgen's .tbl layout (6,000,000 lines at scale 1,
    about 750 MB) parsed into 16 device columns.  ``value``: text bytes per
    second of device time, the text already in HBM (a device tensor; the call's
    device timeline from its first phase to its last, host waits included);
    ``e2e``: the same from pinned host memory, host wall time of the whole call."""
    import numpy as np
    import torch
    from dogqc_b200 import _lib as L
    from dogqc_b200.engine import Engine
    torch.cuda.set_device(local)
    rows = int(6_000_000 * SCALE)
    text, sum_ok, sum_price = tbl_text(rows)
    nbytes = len(text)
    host = torch.frombuffer(bytearray(text), dtype=torch.uint8).pin_memory()
    dev = host.cuda()
    fields = tbl_fields()
    engine = Engine(local)
    for _ in range(args.warmup):
        engine.import_text("lineitem", dev, fields)
    replicas.barrier(world)
    spans, parse = [], []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            n = engine.import_text("lineitem", dev, fields)
            t = engine.import_timing()
            spans.append(t["span_ms"])
            parse.append(t["parse_ms"])
    t = engine.import_timing()
    step_ms = replicas.max_over_ranks(float(np.mean(spans)), world)
    ok = engine.read_column("lineitem", "l_orderkey", L.I32).astype(np.int64).sum()
    price = engine.read_column("lineitem", "l_extendedprice", L.I64).sum()
    parity = bool(n == rows and int(ok) == sum_ok and int(price) == sum_price)
    e2e = []
    for _ in range(max(2, args.steps // 2)):
        engine.import_text("lineitem", host, fields)
        e2e.append(engine.import_timing()["call_ms"])
    e2e_ms = float(np.median(e2e))
    peak, peak_kind = hbm_peak()
    alg = tbl_algorithmic_bytes(nbytes, rows)
    parse_ms = float(np.mean(parse))
    achieved = alg / (parse_ms / 1e3) / 1e9
    out = {
        "metric": "GB/s of .tbl text parsed into device columns (lineitem layout, 16 fields)",
        "value": nbytes * world / (step_ms / 1e3) / 1e9, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded, dbgen layout)",
        "config": {"workload": "tbl_import_lineitem", "rows": rows, "text_bytes": nbytes,
                   "fields": "5 INT, 3 DECIMAL(2), 2 CHAR, 3 DATE, 3 STRING (the reference's lineitem schema)",
                   "l2": "text %.0f MB > L2 (inputs larger than L2)" % (nbytes / 1e6), "parallelism": "replicas"},
        "rows_per_s": rows * world / (step_ms / 1e3),
        "phases_ms": {k: t[k] for k in ("copy_ms", "newline_ms", "line_end_ms", "parse_ms", "string_ms")},
        "parity": parity,
        "e2e": {"value": nbytes / (e2e_ms / 1e3) / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": 8 * (2 + 16), "ms": e2e_ms,
                "how": "dq_table_import_text from pinned host memory, host wall time of the call"},
        "roofline": {"bound": "hbm", "kernel": "imp_parse_kernel", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes": alg, "traffic": load_profile_traffic()},
        "gpu_launches": int(t["kernel_launches"]) * args.steps,
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = tbl_cpu_baseline(fields)
    engine.close()
    return out


def run_served(args, world, rank, local):
    """The served mixed stream at the served configuration: queries of the
    c0-c3 shapes with table sizes log-uniform between 1/100 and 5x of the
    configurations (six sizes per shape, the largest 5x: 300,000,000 c3 fact
    rows; tables preloaded and resident), Poisson arrivals at 100-5,000 queries/s
    through the request server (slots, memory admission against a 150 GB budget,
    continuous batching), against the same streams through a one-slot server
    that runs every request alone and against the requests run one after the
    other as plain plans.  A request of a shape the server has not seen arrives
    in the middle of one stream: its latency (it compiles) and the p99 of the
    others beside it are reported."""
    import threading
    import torch
    from dogqc_b200 import serve
    from dogqc_b200.engine import Engine
    torch.cuda.set_device(local)
    if args.served_sizes == "c4":
        qs = serve.make_c4_queries()
        sizes = {k: [round(x, 4) for x in v] for k, v in serve.c4_sizes().items()}
    else:
        sizes = tuple(float(x) for x in args.served_sizes.split(","))
        qs = serve.make_queries(sizes=sizes)
    engine = Engine(local)
    serve.register(engine, qs)
    rows = {q.index: q.input_rows for q in qs}
    n = 2000
    sched = serve.arrivals(n, None, qs, seed=5)
    _, _, plans = serve.sequence(engine, qs, sched[:len(qs) * 2])
    per, wall1, plans = serve.sequence(engine, qs, sched, plans)
    one = {"queries_per_s": n / wall1, "p50_ms": serve.percentile(per, .5), "p99_ms": serve.percentile(per, .99)}
    for p in plans.values():
        p.free()
    srv = serve.Server(engine, slots=args.slots, batch_max=args.batch_max, batch_rows_max=args.batch_rows_max)
    serve.warm(srv, qs, args.slots, rounds=1)
    runs = []
    with ClockSampler(local) as clocks:
        for _ in range(3):  # closed-loop bursts; the median one is reported
            runs.append(serve.replay(srv, qs, sched))
    infos, wall = sorted(runs, key=lambda r: r[1])[1]
    tot = [i["total_ms"] for i in infos]
    offered = (100, 250, 500, 1000, 2500, 5000)

    def stream(server, rate):
        sch = serve.arrivals(min(4000, max(200, int(rate * 2))), rate, qs, seed=9)
        inf, w = serve.replay(server, qs, sch)
        t = [i["total_ms"] for i in inf]
        return {"offered_qps": rate, "requests": len(sch), "achieved_qps": len(sch) / w,
                "p50_ms": serve.percentile(t, .5), "p99_ms": serve.percentile(t, .99)}
    rates = [stream(srv, r) for r in offered]
    # a cold shape under load: the stream at 1,000 queries/s with and without
    # requests of a shape this server has not prepared (c5, outer join + two
    # aggregations) submitted from another thread 0.5 s into it
    base = stream(srv, 1000)
    cold = {}
    try:
        from dogqc_b200 import workloads
        from dogqc_b200.database import Database, Table
        from dogqc_b200.lowering import Lowering
        from dogqc_b200.relational import RelationalAlgebra
        cdb = workloads.gen_c5(1.0)
        alg = RelationalAlgebra(cdb)
        cplan, ccfg = workloads.build("c5", alg)
        cplan = alg.resolveAlgebraPlan(cplan, ccfg)
        clow = Lowering(cplan)
        for p in clow.pipes:
            if p.table:
                p.table = p.table + "@cold"
        engine.register_database(Database([Table(t.name + "@cold", t.columns, t.types)
                                           for t in cdb.tables.values()]))
        got = {}

        def submit_cold():
            t0 = time.perf_counter()
            tk = srv.submit(clow)
            got["submit_ms"] = (time.perf_counter() - t0) * 1e3
            _, info = srv.wait(tk)
            got["latency_ms"] = (time.perf_counter() - t0) * 1e3
            got["queue_ms"], got["run_ms"] = info["queue_ms"], info["run_ms"]
        th = threading.Timer(0.5, submit_cold)
        th.start()
        with_cold = stream(srv, 1000)
        th.join()
        cold = {"shape": "c5 at 1x (outer join + two aggregations), first sight", "offered_qps": 1000,
                "stream_without": base, "stream_with": with_cold, "cold_request": got}
    except Exception as ex:  # reported, not fatal to the measurement
        cold = {"error": str(ex)}
    st = srv.stats()
    srv.stop()
    # the same Poisson streams one request at a time: one slot, no batching
    srv1 = serve.Server(engine, slots=1, batch_max=1)
    serve.warm(srv1, qs, 1, rounds=1)
    alone = [stream(srv1, r) for r in offered]
    srv1.stop()

    def best_rate(points, p99_ms):  # highest offered rate kept up with at p99 <= p99_ms
        ok = [p["offered_qps"] for p in points
              if p["p99_ms"] <= p99_ms and p["achieved_qps"] >= 0.95 * p["offered_qps"]]
        return max(ok) if ok else 0
    engine.close()
    value = n / wall
    bounds = (5.0, 10.0, 25.0, 50.0)
    return {
        "metric": "queries/s (served mixed stream of c0-c3 queries, closed loop)", "value": value,
        "unit": "queries/s", "n_gpus": world, "steps": n, "warmup": 2, "ms_per_step": wall * 1e3 / n,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded)",
        "config": {"workload": "served_mixed_stream", "shapes": ["c0", "c1", "c2", "c3"], "sizes": sizes,
                   "queries": len(qs), "input_rows_largest": max(rows.values()),
                   "slots": args.slots, "batch_max": args.batch_max or 16,
                   "batch_rows_max": args.batch_rows_max or (1 << 18), "requests": n,
                   "memory_budget_gb": 150, "poisson_qps": list(offered), "parallelism": "replicas"},
        "batches": {"launches": st["batches"], "requests": st["batched"]},
        "p50_ms": serve.percentile(tot, .5), "p99_ms": serve.percentile(tot, .99),
        "one_at_a_time": one, "speedup_vs_one_at_a_time": value / one["queries_per_s"],
        "poisson": rates, "poisson_one_slot_unbatched": alone,
        "max_rate_at_p99": {"%g_ms" % b: {"served": best_rate(rates, b), "one_slot_unbatched": best_rate(alone, b)}
                            for b in bounds},
        "cold_shape": cold,
        "memory_peak_bytes": st["memory_peak"],
        "clocks": clocks.summary(),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--tile-rows", type=int, default=0, help="engine tile size (0: default)")
    ap.add_argument("--ctas-per-sm", type=int, default=0, help="persistent CTAs per SM (0: occupancy)")
    ap.add_argument("--engine-flags", type=int, default=0, help="DQ_CFG_* bits")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="workload size factor (profiling only; the bench line is quoted at 1.0)")
    ap.add_argument("--workload", default="c1", choices=sorted(WORKLOADS) + ["c2x256", "c4", "tbl"],
                    help="c1 (default): the FK-PK join the headline metric is quoted on; c0, c2, c3: "
                         "the other configurations, for the per-pipeline table; c2x256: the batched form; "
                         "c4: the served mixed stream")
    ap.add_argument("--autotune", action="store_true", help="c2x256: pick the batch's tuning by measurement")
    ap.add_argument("--no-stream-bound", action="store_true", help="skip timing the dominant kernel's stream bound")
    ap.add_argument("--tuning", default="", help='plain workloads: a dq_tuning as JSON, e.g. {"rows_per_thread": 2}')
    ap.add_argument("--no-autotune", action="store_true",
                    help="plain workloads: time the plan with the default launch shapes instead of tuning it first")
    ap.add_argument("--slots", type=int, default=4, help="c4: launches in flight on the device (streams)")
    ap.add_argument("--batch-max", type=int, default=0,
                    help="c4: requests of one shape per launch (0: 16; 1: every request alone)")
    ap.add_argument("--batch-rows-max", type=int, default=0,
                    help="c4: requests scanning more input rows run alone (0: 2^18)")
    ap.add_argument("--served-sizes", default="c4",
                    help="c4: 'c4' (the served configuration: six sizes per shape log-uniform in 1/100..5x) or "
                         "a comma-separated list of table sizes, as fractions of the configurations' rows")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    global SCALE, WORKLOAD
    SCALE = args.scale
    WORKLOAD = args.workload
    world, rank, local = dist_setup()
    if args.impl == "ours" and WORKLOAD == "c2x256":
        out = run_batched(args, world, rank, local)
    elif args.impl == "ours" and WORKLOAD == "c4":
        out = run_served(args, world, rank, local)
    elif args.impl == "ours" and WORKLOAD == "tbl":
        out = run_import(args, world, rank, local)
    elif args.impl == "reference" and WORKLOAD not in WORKLOADS:
        out = {"impl": "reference", "unavailable": "the CPU reference arm evaluates plan workloads (c0-c13); "
                                                   "the batched, served and import forms report their own "
                                                   "one-by-one and CPU baselines in the ours line"}
        out = out if rank == 0 else None
    elif args.impl == "reference":
        out = run_reference(args, world, rank)
    else:
        out = run_ours(args, world, rank, local)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    replicas.teardown(world)


if __name__ == "__main__":
    main()
