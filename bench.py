"""Benchmark: Alenka's three-way filter -> join -> group-by -> order pipeline (the
reference README's shape) on seeded tables of lineitem 600M / orders 150M / customer 15M
rows (--scale 10, the default; --scale 1 is the 60M / 15M / 1.5M instance), reported as
fact (lineitem) rows/s.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--scale S]

value: whole-job fact rows/s with every column segment already resident in HBM.
e2e:   the same through the C ABI with host buffers: each step copies the compressed
       segments host->device and the result device->host (alk_session non-resident).
The stored result is checked outside the timed region: against the plain GPU path's,
and against the reference's own stored output for the same tables where one is committed
(tests/golden/ref_ops).
--impl reference: the reference itself (oracle/_ref/alenka_ref: its bison front end and
operators built for the CPU with Thrust's OpenMP backend) on a proportional sample of the
same tables, all host threads, without loading this repository's engine.
N > 1 runs independent replicas (the path does not shard: one GPU per query), timed
as the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fact rows/s filter→join→group-by, bit-exact; batched+learned vs plain; % HBM"
BASE = dict(customers=1_500_000, orders=15_000_000, lineitems=60_000_000)  # --scale 1
SEG_ROWS = 10_000_000
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "alenka_ref")


def sizes(scale):
    return {k: max(1, int(v * scale)) for k, v in BASE.items()}


def _m(n):
    return f"{n / 1e6:g}M"


def workload_config(scale, world):
    """The bench's config, identical in both arms (static: measured figures go elsewhere)."""
    z = sizes(scale)
    return {"workload": ("three-way FILTER->JOIN->JOIN->GROUP BY->ORDER BY ... LIMIT 10 (README shape), "
                         f"lineitem {_m(z['lineitems'])} / orders {_m(z['orders'])} / customer {_m(z['customers'])}, "
                         f"seeded synthetic, FOR-compressed segments of {_m(SEG_ROWS)} rows"),
            "fact_rows_per_step": z["lineitems"], "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (lineitem columns resident, compressed)"}


SEGMENTS = ["AUTOMOBILE", "BUILDING", "FURNITURE", "HOUSEHOLD", "MACHINERY"]


def date_add_days(yyyymmdd, days):
    import datetime
    d = datetime.date(yyyymmdd // 10000, (yyyymmdd // 100) % 100, yyyymmdd % 100) + datetime.timedelta(days=days)
    return d.year * 10000 + d.month * 100 + d.day


def three_way_script(seed, out, limit=10):
    """The README-shaped script with a seed-drawn date and market segment (the text of
    alenka_b200.workloads.three_way_script, built without loading anything)."""
    import random
    r = random.Random(seed * 7919 + 1)
    date = date_add_days(19950702, r.randint(-30, 30))
    seg = SEGMENTS[r.randint(0, 4)]
    lim = f" LIMIT {limit}" if limit else ""
    return (f"OFI := FILTER orders BY o_orderdate < {date};\n"
            f"CF := FILTER customer BY c_mktsegment == \"{seg}\";\n"
            f"LF := FILTER lineitem BY l_shipdate > {date};\n"
            "OLC := SELECT o_orderkey AS o_orderkey, o_orderdate AS o_orderdate, "
            "o_shippriority AS o_shippriority, l_extendedprice AS price, l_discount AS discount "
            "FROM LF JOIN OFI ON l_orderkey = o_orderkey JOIN CF ON o_custkey = c_custkey;\n"
            "F := SELECT o_orderkey AS o_orderkey1, o_orderdate AS orderdate1, o_shippriority AS priority, "
            "SUM(price*(1-discount)) AS sum_revenue, COUNT(o_orderkey) AS cnt "
            "FROM OLC GROUP BY o_orderkey, o_orderdate, o_shippriority;\n"
            "RES := ORDER F BY sum_revenue DESC, orderdate1 ASC;\n"
            f"STORE RES INTO '{out}' USING ('|'){lim};\n")


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader",
                                          "-lms", "200", "-i", str(self.gpu)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1].split()[0]))
                mx.append(float(f[2].split()[0]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


class NvmlClockSampler:
    """SM clock, power and throttle reasons read through NVML every 2 ms during the timed
    region (the region lasts tens of milliseconds, below nvidia-smi's polling period).
    Read-only: no setting of the GPU is changed."""

    def __init__(self, gpu_index):
        import pynvml
        self.n = pynvml
        pynvml.nvmlInit()
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        idx = int(vis.split(",")[gpu_index]) if vis and vis.split(",")[gpu_index].strip().isdigit() else gpu_index
        self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
        self.samples, self.reasons = [], 0
        self.stop_flag = threading.Event()

    def _run(self):
        n = self.n
        while not self.stop_flag.is_set():
            try:
                self.samples.append(n.nvmlDeviceGetClockInfo(self.h, n.NVML_CLOCK_SM))
                self.reasons |= n.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:
                pass
            time.sleep(0.002)

    def start(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def stop(self):
        self.stop_flag.set()
        self.t.join()
        n = self.n
        names = {n.nvmlClocksEventReasonHwSlowdown: "hw_slowdown",
                 n.nvmlClocksEventReasonHwThermalSlowdown: "hw_thermal_slowdown",
                 n.nvmlClocksEventReasonSwThermalSlowdown: "sw_thermal_slowdown",
                 n.nvmlClocksEventReasonSwPowerCap: "sw_power_cap",
                 n.nvmlClocksEventReasonHwPowerBrakeSlowdown: "hw_power_brake_slowdown"}
        try:
            mx = n.nvmlDeviceGetMaxClockInfo(self.h, n.NVML_CLOCK_SM)
        except Exception:
            mx = None
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": mx,
                "reasons": sorted(v for k, v in names.items() if self.reasons & k), "samples": len(self.samples),
                "source": "nvml, 2 ms"}


def clock_sampler(gpu_index):
    try:
        return NvmlClockSampler(gpu_index)
    except Exception:
        return ClockSampler(gpu_index)


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(name):
    """Per-launch DRAM bytes of the hot kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(p):
            if line.strip().startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1].strip())
    except OSError:
        pass
    return None


def profiled_traffic_rows(name):
    """Rows the profiled launch covered, when the summary states them (for scaling)."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(p):
            if line.strip().startswith("traffic_rows_per_launch:"):
                return int(line.split(":")[1].strip())
    except OSError:
        pass
    return None


def scaled_traffic(name, rows):
    """The committed capture's per-launch DRAM bytes scaled to `rows` rows (the stage's
    traffic grows with the rows it scans), or unscaled when the capture states no rows."""
    t, r = profiled_traffic(name), profiled_traffic_rows(name)
    if t is None:
        return None
    return int(t * rows // r) if r else t


def ensure_data(base, scale, seed, writer="engine"):
    """Seeded three-way tables at scale (x60M lineitem rows), written once and reused.
    writer "engine": the engine's generator; "numpy": oracle/refdata.py (the same bytes,
    slower, no engine library loaded)."""
    z = sizes(scale)
    d = os.path.join(base, f"threeway_s{scale}_seed{seed}")
    marker = os.path.join(d, ".complete")
    if not os.path.exists(marker):
        os.makedirs(d, exist_ok=True)
        if writer == "numpy":
            from oracle import refdata
            refdata.three_way(d, z["customers"], z["orders"], z["lineitems"], SEG_ROWS, seed)
        else:
            import alenka_b200 as ab
            ab.gen_three_way(d, z["customers"], z["orders"], z["lineitems"], SEG_ROWS, seed)
        with open(marker, "w") as f:
            f.write(str(z["lineitems"]))
    return d, int(open(marker).read())


def reference_sample_scale(scale):
    """The reference's bounded sample: the same tables scaled down to at most the 60M /
    15M / 1.5M instance, about ten seconds of host work per run."""
    return min(scale, 1.0)


def run_reference_binary(d, script, threads):
    """One run of the reference's own CLI (alenka_ref <script>) in data directory d."""
    p = os.path.join(d, "ref_bench.sql")
    with open(p, "w") as f:
        f.write(script)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    t0 = time.perf_counter()
    r = subprocess.run([REF_BIN, "ref_bench.sql"], cwd=d, env=env, stdout=subprocess.DEVNULL,
                       stderr=subprocess.PIPE, text=True, timeout=3600)
    dt = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed ({r.returncode}): {r.stderr[-300:]}")
    return dt


def cpu_baseline(base, scale, seed, threads):
    """The reference's own operators (oracle/_ref/alenka_ref, Thrust OpenMP backend) on a
    bounded sample; the oracle port when the reference build is absent."""
    sc = reference_sample_scale(scale)
    if os.path.exists(REF_BIN):
        d, rows = ensure_data(base, sc, seed, writer="numpy")
        script = three_way_script(seed, "cpu_q3.txt")
        run_reference_binary(d, script, threads)  # page cache and file images warm
        runs = 2
        dt = sum(run_reference_binary(d, script, threads) for _ in range(runs))
        kind, what = "reference", "the reference's CLI and operators built for the CPU (Thrust OpenMP)"
    else:
        from tests import _oracle
        d, rows = ensure_data(base, sc, seed)
        script = three_way_script(seed, "cpu_q3.txt")
        _oracle.execute(d, script, threads)
        runs = 3
        t0 = time.perf_counter()
        for _ in range(runs):
            _oracle.execute(d, script, threads)
        dt = time.perf_counter() - t0
        kind, what = "port", "the oracle (CPU restatement of the reference operators)"
    z = sizes(sc)
    return {"value": rows * runs / dt, "unit": "rows/s", "cores": threads, "kind": kind,
            "sample": f"{what}: the same script on the same generator's tables at lineitem {_m(z['lineitems'])} / "
                      f"orders {_m(z['orders'])} / customer {_m(z['customers'])} (scale {sc:g} of 60M), "
                      f"{runs} runs, {dt:.2f} s"}


def run_reference(args, rank):
    """--impl reference: the reference's own CLI and operators on the host cores, each step
    one run over a proportional sample of the bench's tables (written by the numpy writer:
    nothing of the engine is loaded). Rank 0 alone runs and prints; other ranks exit."""
    if rank != 0:
        return
    base = args.data_dir or os.path.join(tempfile.gettempdir(), "alenka_bench_ref")
    threads = os.cpu_count() or 1
    sc = reference_sample_scale(args.scale)
    z = sizes(sc)
    script = three_way_script(args.seed, "ref_q3.txt")
    if not os.path.exists(REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/alenka_ref absent "
                                                              "(oracle/build_ref.sh needs the reference sources)"}))
        return
    d, rows = ensure_data(base, sc, args.seed, writer="numpy")
    for _ in range(args.warmup):
        run_reference_binary(d, script, threads)
    dt = sum(run_reference_binary(d, script, threads) for _ in range(args.steps))
    value = rows * args.steps / dt
    sample = (f"each step one run of the reference's CLI over lineitem {_m(z['lineitems'])} / orders "
              f"{_m(z['orders'])} / customer {_m(z['customers'])} (the same generator, scale {sc:g} of 60M)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1000 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": workload_config(args.scale, args.gpus),
        "implementation": "reference sources (bison front end, operators, codec) built for the CPU with Thrust's "
                          "OpenMP device system; moderngpu's inner_join/segreduce/reduce restated on the host "
                          "(oracle/ref_shim), the reference does not vendor moderngpu",
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def timed_steps(sess, script, steps, torch, dist):
    """K executions bracketed by a barrier + synchronize, timed with CUDA events on the
    session's stream; returns (ms per step (max over ranks), stats summed over steps)."""
    stream = torch.cuda.ExternalStream(sess.stream)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    acc = {"kernels": 0, "h2d": 0, "d2h": 0, "rows": 0, "hot_ms": 0.0, "hot_bytes": 0, "hot_launches": 0, "plan": 0,
           "query_dev_ms": 0.0}
    for _ in range(steps):
        sess.execute(script)
        st = sess.stats()
        acc["kernels"] += st.kernels
        acc["h2d"] += st.h2d_bytes
        acc["d2h"] += st.d2h_bytes
        acc["rows"] += st.rows_scanned
        acc["hot_ms"] += st.hot_kernel_ms
        acc["hot_bytes"] += st.hot_kernel_bytes
        acc["hot_launches"] += st.hot_kernel_launches
        acc["plan"] = st.plan
        acc["query_dev_ms"] += st.query_device_ms
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    if dist:
        ms = max_over_ranks(ms, dist, torch, "cuda")
    return ms, acc


def max_over_ranks(ms, dist, torch, device):
    """The slowest rank's milliseconds: every replica's step must be done for the job's."""
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _steps(sess, fn, steps, torch):
    """steps calls of fn bracketed by synchronize, timed with CUDA events on the session's
    stream; returns (ms per step, summed stats)."""
    stream = torch.cuda.ExternalStream(sess.stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    acc = {"kernels": 0, "hot_ms": 0.0, "hot_bytes": 0, "hot_launches": 0, "plan": 0, "rows": 0}
    for _ in range(steps):
        fn()
        st = sess.stats()
        acc["kernels"] += st.kernels
        acc["hot_ms"] += st.hot_kernel_ms
        acc["hot_bytes"] += st.hot_kernel_bytes
        acc["hot_launches"] += st.hot_kernel_launches
        acc["plan"] = st.plan
        acc["rows"] += st.rows_scanned
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, acc


def run_batched(args, torch):
    """Many queries of the single-table filter + group-by family over tables generated in
    device memory (lognormal segment sizes), one batch per step; beside it the same
    scripts one at a time on the dense path and on the plain operator path."""
    import alenka_b200 as ab
    from alenka_b200 import workloads as wl
    total = int(6_000_000_000 * args.scale)
    layout = [t for t in wl.batched_layout(args.queries, total, args.seed) if t]
    rows = sum(sum(t) for t in layout)
    d = tempfile.mkdtemp(prefix="alenka_batched_")
    sess = ab.Session(d, resident=True)
    if args.no_autotune:
        sess.tuning(autotune=False)
    if args.launch_shape:
        sess.set_tuning(tuple(int(v) for v in args.launch_shape.split(",")))
    t0 = time.perf_counter()
    for q, segs in enumerate(layout):
        sess.gen_flat_resident(f"li{q:03d}", segs, args.seed * 1000 + q)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    scripts = [wl.flat_script(args.seed * 1000 + q, out=f"bq{q:03d}.txt", table=f"li{q:03d}")
               for q in range(len(layout))]
    for _ in range(args.warmup):
        sess.execute_batch(scripts)
    sess.set_timing(True)
    clk = clock_sampler(0)
    clk.start()
    ms, acc = _steps(sess, lambda: sess.execute_batch(scripts), args.steps, torch)
    clocks = clk.stop()
    sess.set_timing(False)
    tuning = sess.tuning()
    host_ms = list(sess.stats().batch_host_ms)
    one_ms = plain_ms = float("nan")
    if not args.batched_only:
        for sc in scripts[:4]:
            sess.execute(sc)
        one_ms, _ = _steps(sess, lambda: [sess.execute(sc) for sc in scripts], 1, torch)
        sess.set_plain(True)
        for sc in scripts[:2]:
            sess.execute(sc)
        plain_ms, _ = _steps(sess, lambda: [sess.execute(sc) for sc in scripts], 1, torch)
    sess.close()
    peak, peak_kind = measured_peak_hbm()
    hot = None
    if acc["hot_launches"]:
        pl_bytes = acc["hot_bytes"] / acc["hot_launches"]
        pl_ms = acc["hot_ms"] / acc["hot_launches"]
        achieved = pl_bytes / (pl_ms / 1000.0) / 1e9
        hot = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
               "traffic": (profiled_traffic("batched_groupby_flat.md") * rows // profiled_traffic_rows(
                   "batched_groupby_flat.md")) if profiled_traffic_rows("batched_groupby_flat.md") else None,
               "traffic_note": "ncu capture at 120M rows, scaled by rows to this batch",
               "kernel": "k_gb_tma (batched filter + dense group-by, one launch per batch)",
               "algorithmic_bytes": "scanned rows x stored widths of the columns the queries read",
               "algorithmic_bytes_per_launch": int(pl_bytes), "avg_launch_ms": pl_ms,
               "peak_source": f"{peak_kind} hbm_gbs"}
    print(json.dumps({
        "metric": "fact rows/s, batched filter + group-by (single-table family)", "value": rows / (ms / 1000.0),
        "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (generated in device memory)",
        "config": {"workload": f"{len(layout)} queries over {rows} lineitem rows in "
                               f"{sum(len(t) for t in layout)} lognormal segments (median 4M, 1M-32M)",
                   "launch_shape": {"consumer_warps": tuning[0], "stages": tuning[1], "blocks_per_sm": tuning[2]},
                   "one_at_a_time_dense_rows_per_s": rows / (one_ms / 1000.0),
                   "plain_gpu_rows_per_s": rows / (plain_ms / 1000.0),
                   "batched_vs_plain": plain_ms / ms, "generation_s": gen_s,
                   "host_ms_plan_launch_finish": host_ms, "l2": "inputs larger than L2"},
        "e2e": None, "gpu_launches": acc["kernels"], "roofline": hot, "cpu_baseline": None, "clocks": clocks,
    }), flush=True)


def run_groupby_high(args, torch):
    """High-cardinality group-by over a lineitem-shaped table generated in device memory
    (600M rows): FILTER lineitem BY l_shipdate < d, then GROUP BY l_orderkey (rows in key
    order, 4 rows per key, ~150M keys) and GROUP BY l_extendedprice, l_discount (unsorted,
    ~95M groups). Each is timed in its fused hash form (filter and hashing in one pass),
    its sort-based form (the sort runs for the unsorted keys and is skipped for the
    ordered ones), and the form the engine picks."""
    import alenka_b200 as ab
    from alenka_b200 import workloads as wl
    rows = int(600_000_000 * args.scale)
    seg = 10_000_000
    segs = [seg] * (rows // seg) + ([rows % seg] if rows % seg else [])
    d = tempfile.mkdtemp(prefix="alenka_gbhigh_")
    sess = ab.Session(d, resident=True)
    sess.gen_flat_resident("lineitem", segs, args.seed)
    cut = wl.flat_cutoff(args.seed)
    scripts = {
        "key_order": (f"LF := FILTER lineitem BY l_shipdate < {cut};\n"
                      "R := SELECT l_orderkey AS k, SUM(l_quantity) AS q, SUM(l_extendedprice*(1-l_discount)) AS rev, "
                      "COUNT(l_orderkey) AS c FROM LF GROUP BY l_orderkey;\n"
                      "STORE R INTO 'gbh.txt' USING ('|');\n"),
        "unsorted": (f"LF := FILTER lineitem BY l_shipdate < {cut};\n"
                     "R := SELECT l_extendedprice AS p, l_discount AS d, SUM(l_quantity) AS q, "
                     "COUNT(l_orderkey) AS c FROM LF GROUP BY l_extendedprice, l_discount;\n"
                     "STORE R INTO 'gbu.txt' USING ('|');\n"),
    }
    out = {}
    steps = max(1, args.steps // 8)
    for sname, script in scripts.items():
        outs = {}
        for name, mode in (("auto", 0), ("hash", 1), ("sort", 2)):
            sess.set_groupby(mode)
            sess.execute(script)
            sess.set_timing(True)
            ms, acc = _steps(sess, lambda: sess.execute(script), steps, torch)
            sess.set_timing(False)
            gb_ms = acc["hot_ms"] / max(1, acc["hot_launches"])
            st = sess.stats()
            outs[name] = {"ms_per_query": ms, "rows_per_s": rows / (ms / 1000.0), "groupby_ms": gb_ms,
                          "groupby_rows_per_s": rows / (gb_ms / 1000.0) if gb_ms else None,
                          "form": "sort" if st.sort_groupbys else ("fused hash" if st.hash_groupbys else "other")}
        out[sname] = outs
        with open(os.path.join(d, "gbh.txt" if sname == "key_order" else "gbu.txt"), "rb") as f:
            f.seek(0, 2)
            outs["stored_bytes"] = f.tell()
    sess.close()
    best = min(out["unsorted"]["hash"]["groupby_ms"], out["unsorted"]["sort"]["groupby_ms"])
    print(json.dumps({"metric": "fact rows/s, filter + GROUP BY (high cardinality), group-by device time",
                      "value": rows / (best / 1000.0), "unit": "rows/s", "n_gpus": 1, "dtype": "int64",
                      "data": "synthetic (generated in device memory)",
                      "config": {"workload": f"lineitem {rows} rows, {len(segs)} segments; GROUP BY l_orderkey "
                                             f"(~{rows // 4} keys, key order) and GROUP BY l_extendedprice, "
                                             "l_discount (unsorted)",
                                 "forms": out}}), flush=True)


def run_encode(args, torch):
    """The segment writer behind STORE ... BINARY: a lineitem-shaped result of 60M rows and
    five numeric columns (l_orderkey in order, l_quantity, l_extendedprice, l_discount,
    l_shipdate) encoded into segment images of 10M rows per column, FOR or FOR-delta as the
    reference's delta switch picks. One step is one call of the batched device writer
    (alk_encode_segments_device, mode 2) over every segment of every column; e2e adds the
    upload of the values from pinned host memory and the download of every image."""
    import ctypes
    import numpy as np
    import alenka_b200 as ab
    L = ab.lib()
    L.alk_encode_segment_device.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p]
    L.alk_encode_segment.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    vp = ctypes.c_void_p
    L.alk_encode_segments_device.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_int, vp, vp, vp, vp]
    rows = int(60_000_000 * args.scale)
    seg = min(10_000_000, rows)
    g = torch.Generator(device="cuda")
    g.manual_seed(args.seed)

    def rnd(lo, hi):
        return torch.randint(lo, hi + 1, (rows,), device="cuda", generator=g, dtype=torch.int64)
    cols = {"l_orderkey": torch.cumsum(rnd(0, 1), 0) * 4 + 1, "l_quantity": rnd(1, 50),
            "l_extendedprice": rnd(90_000, 10_500_000), "l_discount": rnd(0, 10),
            "l_shipdate": rnd(19_920_102, 19_981_201)}
    segs = [(c, s0, min(seg, rows - s0)) for c in cols for s0 in range(0, rows, seg)]
    k = len(segs)
    cap = (24 + 8 * seg + 32 + 255) // 256 * 256
    imgs = torch.empty(k * cap // 8, dtype=torch.int64, device="cuda")
    ln = ctypes.c_size_t()
    P = ctypes.c_void_p * k
    d_imgs = P(*[imgs.data_ptr() + i * cap for i in range(k)])
    counts = (ctypes.c_uint32 * k)(*[n for _, _, n in segs])
    caps = (ctypes.c_size_t * k)(*([cap] * k))
    lens = (ctypes.c_size_t * k)()

    def encode(src):
        rc = L.alk_encode_segments_device(src, counts, k, 2, d_imgs, caps, lens, None)
        if rc:
            raise RuntimeError(f"segment writer: status {rc}")
        return sum(lens)
    src_dev = P(*[cols[c].data_ptr() + 8 * s0 for c, s0, _ in segs])

    def step():
        return encode(src_dev)
    args.warmup = max(args.warmup, 3)
    for _ in range(args.warmup):
        img_bytes = step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = clock_sampler(0)
    clk.start()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / args.steps
    in_bytes = 8 * rows * len(cols)
    alg = in_bytes + img_bytes
    # end to end: values from pinned host memory, every image back to pinned host memory
    host_cols = {c: t.cpu().pin_memory() for c, t in cols.items()}
    stage = {c: torch.empty_like(t) for c, t in cols.items()}
    src_stage = P(*[stage[c].data_ptr() + 8 * s0 for c, s0, _ in segs])
    host_img = torch.empty(k * cap, dtype=torch.uint8).pin_memory()
    img_u8 = imgs.view(torch.uint8)

    def e2e_step():
        for c in cols:
            stage[c].copy_(host_cols[c], non_blocking=True)
        encode(src_stage)
        for i in range(k):
            host_img[i * cap:i * cap + lens[i]].copy_(img_u8[i * cap:i * cap + lens[i]], non_blocking=True)
        torch.cuda.synchronize()
    e2e_step()
    e2e_steps = max(1, args.steps // 2)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(e2e_steps):
        e2e_step()
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    cpu = None
    if not args.no_cpu_baseline:  # the host writer (pinned to the reference's own files), one core
        n_cpu = min(rows, 4_000_000)
        sample = {c: np.ascontiguousarray(host_cols[c][:n_cpu].numpy()) for c in cols}
        out = ctypes.create_string_buffer(24 + 8 * n_cpu + 64)
        t0 = time.perf_counter()
        for c in cols:
            v = sample[c]
            rc = L.alk_encode_segment(v.ctypes.data, n_cpu, 1, out, len(out), ctypes.byref(ln))
            if rc:
                raise RuntimeError(f"host segment writer: status {rc}")
        dt = time.perf_counter() - t0
        cpu = {"value": n_cpu / dt, "unit": "rows/s", "cores": 1, "kind": "port",
               "sample": f"{n_cpu} rows x {len(cols)} columns, one segment per column (host writer)"}
    peak, peak_kind = measured_peak_hbm()
    achieved = alg / (ms / 1000.0) / 1e9
    traffic = profiled_traffic("encode_segment_lineitem.md")
    trows = profiled_traffic_rows("encode_segment_lineitem.md")
    print(json.dumps({
        "metric": "rows/s written as segment images (STORE BINARY of 5 numeric lineitem columns)",
        "value": rows / (ms / 1000.0), "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded, generated in device memory)",
        "config": {"workload": f"{rows} rows x {len(cols)} columns in segments of {seg} rows "
                               f"({len(segs)} segment images, {img_bytes} bytes)",
                   "l2": "inputs larger than L2"},
        "e2e": {"value": rows / (e2e_ms / 1000.0), "unit": "rows/s", "h2d_bytes_per_step": in_bytes,
                "d2h_bytes_per_step": img_bytes},
        "gpu_launches": 4 * args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (traffic * rows // trows) if traffic and trows else None,
                     "traffic_note": "ncu capture of one step at a smaller size, scaled by rows",
                     "kernel": "k_enc_stats_batch + k_enc_pack_batch (the whole step: 4 launches, 1 synchronisation)",
                     "algorithmic_bytes": "8 B per value read + the image bytes written",
                     "algorithmic_bytes_per_step": alg, "peak_source": f"{peak_kind} hbm_gbs"},
        "cpu_baseline": cpu, "clocks": clocks,
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--scale", type=float, default=None,
                    help="three_way: x60M lineitem rows (default 10: 600M / 150M / 15M); other workloads: x their own base (default 1)")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--data-dir", default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fused-only", action="store_true",
                    help="time only the resident fused plan (profiling runs)")
    ap.add_argument("--workload", default="three_way",
                    choices=["three_way", "batched", "groupby_high", "encode", "compressed", "estimator", "load",
                             "star"],
                    help="three_way: the filter -> join -> group-by pipeline (default); batched: many "
                         "single-table filter + group-by queries per step; compressed: the three-way on "
                         "FOR-delta tables with Zipf(1.1) join keys")
    ap.add_argument("--queries", type=int, default=256)
    ap.add_argument("--batched-only", action="store_true", help="batched workload: skip the one-at-a-time runs")
    ap.add_argument("--no-autotune", action="store_true", help="batched workload: default launch shape")
    ap.add_argument("--launch-shape", default=None,
                    help="batched workload: fixed launch shape 'consumer_warps,stages,blocks_per_sm'")
    ap.add_argument("--no-graphs", action="store_true",
                    help="run every query without CUDA-graph replay (same kernels; for ncu, whose per-kernel "
                         "replay does not handle graph memory nodes)")
    args = ap.parse_args()
    if args.scale is None:
        args.scale = 10.0 if args.workload in ("three_way", "compressed", "star") else 1.0
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        if args.workload == "star":
            if rank == 0:
                run_reference_star(args)
            return
        run_reference(args, rank)
        return
    import torch
    torch.cuda.set_device(local)
    if args.workload in ("batched", "groupby_high", "encode", "compressed", "estimator", "load", "star"):
        if rank == 0:
            {"batched": run_batched, "groupby_high": run_groupby_high, "encode": run_encode,
             "compressed": run_compressed, "estimator": run_estimator, "load": run_load,
             "star": run_star}[args.workload](args, torch)
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    run_three_way(args, torch, dist, world, rank, local)


def golden_output(scale, seed):
    """The reference's own stored output for this instance, when one is committed."""
    try:
        m = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_ops", "manifest.json")))
    except OSError:
        return None, None
    want = three_way_script(seed, "q3.txt")
    z = sizes(scale)
    for c in m["cases"]:
        ds = m["datasets"][c["dataset"]]
        if (c["script"] == want and ds.get("kind") == "three_way" and ds["rows"] == z["lineitems"]
                and ds["orders"] == z["orders"] and ds["customers"] == z["customers"]
                and ds["seg_rows"] == SEG_ROWS and ds["seed"] == seed and "file" in c):
            return c["name"], open(os.path.join(ROOT, "tests", "golden", "ref_ops", c["file"]), "rb").read()
    return None, None


def query_bytes(d, fact_rows, counts):
    """Algorithmic bytes of one query (the scope table's B): every referenced column at its
    stored width over the scanned rows, plus 32 B per probe into, and 64 B per aggregate
    update of, a table larger than L2, plus 32 B per build row, plus the output."""
    import struct
    cols = {"lineitem": ["l_orderkey", "l_shipdate", "l_extendedprice", "l_discount"],
            "orders": ["o_orderkey", "o_custkey", "o_orderdate", "o_shippriority"],
            "customer": ["c_custkey", "c_mktsegment"]}
    total = 0
    for t, cs in cols.items():
        for c in cs:
            g = 0
            while True:
                p = os.path.join(d, f"{t}.{c}.{g}")
                if not os.path.exists(p):
                    p += ".idx"
                if not os.path.exists(p):
                    break
                with open(p, "rb") as f:
                    total += struct.unpack("<I", f.read(4))[0]  # payload bytes at the stored width
                g += 1
    return total + 32 * counts.get("probe_rows_beyond_l2", 0) + 64 * counts.get("agg_rows_beyond_l2", 0) \
        + 32 * counts.get("build_rows", 0) + counts.get("output_bytes", 0)


def run_estimator(args, torch):
    """The learned estimator at the config-2 scale: three-way tables of 60M / 15M / 1.5M
    rows in 1M-row segments, seeded queries of the README shape in record mode until about
    100k exact (query, segment) records exist, training on the device, then the q-error
    of held-out records (rows passing filter and probe per segment) for the network and
    for the classical histogram / independence estimate, and the bytes that 12 new
    queries' first runs reserve with and without the estimator (results identical)."""
    import numpy as np
    import alenka_b200 as ab
    from alenka_b200 import workloads as wl
    base = args.data_dir or os.path.join(tempfile.gettempdir(), "alenka_bench")
    d = os.path.join(base, f"estimator_seed{args.seed}")
    marker = os.path.join(d, ".complete")
    if not os.path.exists(marker):
        os.makedirs(d, exist_ok=True)
        wl.make_three_way(d, scale=1.0, seg_rows=1_000_000, seed=args.seed)
        open(marker, "w").close()

    def run(s, script):
        try:
            s.execute(script)
        except ab.AlenkaError as e:  # an empty join stops the reference with an error too
            return "error: " + str(e)
        return None
    want_records, n_test = 100_000, 300
    epochs = 120  # held-out p95 q-error at this scale: 56.9 after 40 epochs, 37.9 after 120, 84.5 after 300
    t0 = time.perf_counter()
    with ab.Session(d) as s:
        s.card_mode(record=True)
        q = 0
        while q < 20_000:  # about 100k records; a bound in case the queries skip most segments
            run(s, wl.card_script(q, out="qc.txt"))
            q += 1
            if q % 50 == 0 and len(s.card_records()[1]) >= want_records:
                break
        n_train = q
        split = len(s.card_records()[1])
        for k in range(n_test):
            run(s, wl.card_script(n_train + k, out="qc.txt"))
        record_s = time.perf_counter() - t0
        x, y, m = s.card_records()
        t1 = time.perf_counter()
        l_first = s.card_train(0, split, epochs=1, batch=256, lr=1e-3, seed=3)
        l_last = s.card_train(0, split, epochs=epochs, batch=256, lr=1e-3, seed=4)
        train_s = time.perf_counter() - t1
        xt, yt, mt = x[split:], y[split:], m[split:]
        pt = np.minimum(s.card_predict(xt), 0.0)
        rows = np.exp2(xt[:, 3] * 32) - 1
        floor = np.log(0.5 / np.maximum(rows, 1))
        act = yt[:, 0] + yt[:, 1] * mt[:, 1]
        est = pt[:, 0] + pt[:, 1] * mt[:, 1]
        classical = np.maximum(np.log(np.maximum(xt[:, 9] * np.where(mt[:, 1] > 0, xt[:, 10], 1.0), 1e-30)), floor)
        q_mlp, q_cls = np.exp(np.abs(est - act)), np.exp(np.abs(classical - act))
        first = {}
        outs = {}
        for use in (False, True):
            s.card_mode(record=False, use=use)
            res, tot, reruns = [], 0, 0
            for k in range(100_000, 100_012):
                s.card_forget()
                err = run(s, wl.card_script(k, out="qc.txt"))
                st = s.stats()
                tot += st.reserved_bytes
                reruns += st.card_reruns
                with open(os.path.join(d, "qc.txt"), "rb") as f:
                    res.append(err or f.read())
            outs[use] = res
            first["with_estimator" if use else "upper_bound"] = {"reserved_mib": tot / 2**20, "reruns": reruns}
    if outs[True] != outs[False]:
        raise SystemExit("bench: estimator sizing changed a result")
    print(json.dumps({
        "metric": "q-error of the learned cardinality estimate (rows passing filter and probe per query segment)",
        "value": float(np.median(q_mlp)), "unit": "q-error (median)", "higher_is_better": False, "n_gpus": 1,
        "data": "synthetic", "dtype": "bf16 weights, fp32 accumulate",
        "config": {"workload": "three-way tables 60M / 15M / 1.5M in 1M-row segments (config-2 scale); "
                               "seeded README-shape queries with varied operators and constants",
                   "train_queries": n_train, "train_records": int(split), "test_queries": n_test,
                   "test_records": int(len(act))},
        "q_error": {"mlp": {"median": float(np.median(q_mlp)), "p95": float(np.percentile(q_mlp, 95)),
                            "max": float(q_mlp.max())},
                    "classical": {"median": float(np.median(q_cls)), "p95": float(np.percentile(q_cls, 95)),
                                  "max": float(q_cls.max())}},
        "loss": {"first_epoch": l_first, "last_epoch": l_last},
        "seconds": {"record": record_s, "train": train_s},
        "first_runs": first, "verified": {"results_identical": True}}), flush=True)


def run_load(args, torch):
    """The text loader: a lineitem-shaped table (60M rows x scale, generated in device
    memory) is stored as a '|'-separated text file, then each step LOADs it (the file read
    from the page cache, copied to the device and parsed there: integers, decimals, char
    columns) and the device part of the load is timed with CUDA events on the session's
    stream; e2e is the whole LOAD statement's wall time."""
    import alenka_b200 as ab
    rows = int(60_000_000 * args.scale)
    seg = 10_000_000
    segs = [seg] * (rows // seg) + ([rows % seg] if rows % seg else [])
    d = tempfile.mkdtemp(prefix="alenka_load_")
    with ab.Session(d, resident=True) as s:
        s.gen_flat_resident("lineitem", segs, args.seed)
        s.execute("STORE lineitem INTO 'lineitem.tbl' USING ('|');\n")
    nbytes = os.path.getsize(os.path.join(d, "lineitem.tbl"))
    script = ("T := LOAD 'lineitem.tbl' USING ('|') AS (k{1}:int, q{2}:int, p{3}:decimal(12,2), "
              "dc{4}:decimal(4,2), sd{5}:int, rf{6}:varchar(1), ls{7}:varchar(1));\n")
    sess = ab.Session(d, resident=True)
    for _ in range(max(1, args.warmup)):
        sess.execute(script)
    stream = torch.cuda.ExternalStream(sess.stream)
    steps = max(1, args.steps // 4)
    walls, devs = [], []
    for _ in range(steps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        sess.execute(script)
        e1.record(stream)
        torch.cuda.synchronize()
        walls.append((time.perf_counter() - t0) * 1000.0)
        devs.append(e0.elapsed_time(e1))
    sess.close()
    wall = statistics.median(walls)
    # beside it: the reference's own LOAD + STORE BINARY (built for the CPU) on the file's
    # first 2M records, the bounded sample
    cpu = None
    if os.path.exists(REF_BIN) and not args.no_cpu_baseline:
        rd = os.path.join(d, "ref")
        os.makedirs(rd, exist_ok=True)
        sample = 2_000_000
        with open(os.path.join(d, "lineitem.tbl"), "rb") as src, open(os.path.join(rd, "lineitem.tbl"), "wb") as dst:
            for k, line in enumerate(src):
                if k == sample:
                    break
                dst.write(line)
        ref_script = script + "STORE T INTO 'tl' BINARY;\n"
        threads = os.cpu_count() or 1
        run_reference_binary(rd, ref_script, threads)  # page cache warm
        dt = run_reference_binary(rd, ref_script, threads)
        cpu = {"value": sample / dt, "unit": "rows/s", "cores": threads, "kind": "reference",
               "sample": f"the reference's CLI built for the CPU: LOAD + STORE BINARY of the file's first {sample} "
                         f"records, {dt:.2f} s (the engine's figure above is the LOAD alone)"}
    print(json.dumps({
        "metric": "text loader: fact rows/s parsed (LOAD ... USING ('|') AS (...))", "value": rows / (wall / 1000.0),
        "unit": "rows/s", "n_gpus": 1, "steps": steps, "higher_is_better": True, "dtype": "int64 / char",
        "data": "synthetic (a device-generated lineitem shape stored as text)",
        "config": {"workload": f"lineitem text, {rows} rows, {nbytes} bytes, 7 columns (2 int, 2 decimal, 1 "
                               "yyyymmdd int, 2 char(1))"},
        "ms_per_load": wall, "text_gb_per_s": nbytes / (wall / 1000.0) / 1e9,
        "note": "the LOAD statement end to end: file read from the page cache, host newline count, copy to the "
                "device, newline positions and the parse on the device",
        "cpu_baseline": cpu}), flush=True)


def run_compressed(args, torch):
    """The compressed and skewed config: the three-way tables stored FOR-delta (every
    integer column; the engine keeps them resident re-encoded as FOR at each segment's
    narrowest width) with lineitem's orderkeys Zipf(1.1) over the orders, in key order.
    The fused plan is timed and checked against the operator-at-a-time path; the oracle
    parity of this shape is a GPU test at a smaller scale."""
    import alenka_b200 as ab
    base = args.data_dir or os.path.join(tempfile.gettempdir(), "alenka_bench")
    scale = args.scale
    z = sizes(scale)
    d = os.path.join(base, f"compressed_s{scale}_seed{args.seed}")
    marker = os.path.join(d, ".complete")
    if not os.path.exists(marker):
        os.makedirs(d, exist_ok=True)
        ab.gen_three_way(d, z["customers"], z["orders"], z["lineitems"], SEG_ROWS, args.seed, delta=True, zipf=1.1)
        with open(marker, "w") as f:
            f.write(str(z["lineitems"]))
    rows = z["lineitems"]
    out_name = "bench_q5.txt"
    script = three_way_script(args.seed, out_name)
    args.warmup = max(args.warmup, 3)
    sess = ab.Session(d, resident=True, graphs=not args.no_graphs)
    for t in ("lineitem", "orders", "customer"):
        sess.preload(t)
    for _ in range(args.warmup):
        sess.execute(script)
    sess.set_timing(True)
    clk = clock_sampler(0)
    clk.start()
    ms, acc = timed_steps(sess, script, args.steps, torch, None)
    clocks = clk.stop()
    sess.set_timing(False)
    sess.close()
    fused_out = open(os.path.join(d, out_name), "rb").read()
    plain = ab.Session(d, resident=True, plain=True)
    plain.execute(script)
    pms, _ = timed_steps(plain, script, 3, torch, None)
    plain.close()
    plain_out = open(os.path.join(d, out_name), "rb").read()
    if fused_out != plain_out:
        raise SystemExit("bench: compressed config, fused and operator paths differ")
    dev_ms = acc["query_dev_ms"] / args.steps
    peak, peak_kind = measured_peak_hbm()
    qb = query_bytes(d, rows, {})
    print(json.dumps({
        "metric": METRIC + " (compressed + skewed config)", "value": rows / (ms / 1000.0), "unit": "rows/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "dtype": "int64", "data": "synthetic",
        "config": {"workload": f"three-way FILTER->JOIN->JOIN->GROUP BY->ORDER BY ... LIMIT 10, lineitem "
                               f"{rows} / orders {z['orders']} / customer {z['customers']}, every integer column "
                               "FOR-delta on disk, l_orderkey Zipf(1.1) over the orders in key order",
                   "segment_rows": SEG_ROWS},
        "plan": {0: "operator-at-a-time", 1: "fused", 2: "fused, replayed from its CUDA graph"}.get(acc["plan"], "?"),
        "device_ms_per_step": dev_ms, "plain_ms_per_step": pms, "fused_vs_plain": pms / ms,
        "verified": {"fused_eq_plain": True},
        "gpu_launches": acc["kernels"],
        "query_roofline": {"bytes_per_query": qb, "bytes": "every referenced column over all rows at its on-disk "
                           "(FOR-delta packed) width; the scans read the resident FOR re-encoding, wider",
                           "achieved": qb / (dev_ms / 1000.0) / 1e9, "peak": peak, "unit": "GB/s",
                           "frac": qb / (dev_ms / 1000.0) / 1e9 / peak, "peak_source": peak_kind},
        "clocks": clocks}), flush=True)


STAR_METRIC = "fact rows/s, star join through a bitmap join index + GROUP BY + ORDER BY ... LIMIT 10"


def star_scripts(seed, out):
    """The star workload's CREATE INDEX and its query: lineitem indexed on
    orders.o_orderdate, joined with orders filtered on ten seed-drawn dates, grouped by
    date, ordered by revenue, top 10."""
    import random
    r = random.Random(seed * 31 + 7)
    dates = sorted({date_add_days(19920101, r.randint(0, 2400)) for _ in range(10)})
    setup = ("CREATE INDEX lo ON lineitem(orders.o_orderdate) FROM lineitem, orders "
             "WHERE lineitem.l_orderkey = orders.o_orderkey;\n")
    script = ("OF := FILTER orders BY " + " OR ".join(f"o_orderdate == {x}" for x in dates) + ";\n"
              "J := SELECT l_orderkey AS l_orderkey, l_extendedprice AS l_extendedprice, o_orderdate AS o_orderdate "
              "FROM lineitem JOIN OF ON l_orderkey = o_orderkey;\n"
              "G := SELECT o_orderdate AS odate, SUM(l_extendedprice) AS rev, COUNT(l_orderkey) AS cnt "
              "FROM J GROUP BY o_orderdate;\n"
              "R := ORDER G BY rev DESC;\n"
              f"STORE R INTO '{out}' USING ('|') LIMIT 10;\n")
    return setup, script, dates


def star_config(scale, seed):
    z = sizes(scale)
    _, _, dates = star_scripts(seed, "x")
    return {"workload": f"lineitem {z['lineitems']} rows in segments of {z['orders']} / orders {z['orders']} / "
                        f"customer {z['customers']}, one segment each; lineitem indexed on orders.o_orderdate; star "
                        f"join with orders filtered on {len(dates)} dates, GROUP BY date, ORDER BY revenue DESC "
                        "LIMIT 10",
            "dates": dates}


def star_reference(base, scale, seed, threads, steps, warmup):
    """The reference's own CLI (oracle/_ref/alenka_ref, Thrust OpenMP) on the star workload's
    tables at a bounded scale, written by the numpy writer (nothing of the engine loaded):
    CREATE INDEX once, then `steps` runs of the query. Returns (seconds of CREATE INDEX,
    seconds per query, fact rows, sample text)."""
    from oracle import refdata
    z = sizes(scale)
    d = os.path.join(base, f"star_numpy_s{scale}_seed{seed}")
    marker = os.path.join(d, ".complete")
    if not os.path.exists(marker):
        os.makedirs(d, exist_ok=True)
        refdata.three_way(d, z["customers"], z["orders"], z["lineitems"], z["orders"], seed)
        with open(marker, "w") as f:
            f.write(str(z["lineitems"]))
    setup, script, _ = star_scripts(seed, "ref_star.txt")
    index_s = run_reference_binary(d, setup, threads)
    for _ in range(warmup):
        run_reference_binary(d, script, threads)
    dt = sum(run_reference_binary(d, script, threads) for _ in range(steps)) / steps
    sample = (f"the reference's CLI and operators built for the CPU (Thrust OpenMP): CREATE INDEX once, then the "
              f"star query over lineitem {_m(z['lineitems'])} / orders {_m(z['orders'])} / customer "
              f"{_m(z['customers'])} (the same generator, scale {scale:g} of the 60M instance), {steps} runs, "
              f"{dt * steps:.2f} s")
    return index_s, dt, z["lineitems"], sample


def run_reference_star(args):
    """--impl reference --workload star: the reference's own star join on the host cores."""
    threads = os.cpu_count() or 1
    if not os.path.exists(REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/alenka_ref absent "
                                                              "(oracle/build_ref.sh needs the reference sources)"}))
        return
    base = args.data_dir or os.path.join(tempfile.gettempdir(), "alenka_bench_ref")
    sc = reference_sample_scale(args.scale)
    index_s, dt, rows, sample = star_reference(base, sc, args.seed, threads, args.steps, args.warmup)
    value = rows / dt
    print(json.dumps({
        "impl": "reference", "metric": STAR_METRIC, "value": value, "unit": "rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1000, "higher_is_better": True,
        "dtype": "int64", "data": "synthetic", "config": star_config(args.scale, args.seed),
        "create_index": {"seconds": index_s, "rows_per_s": rows / index_s},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_star(args, torch):
    """Star join through a bitmap join index at the headline fact size: lineitem 600M rows in
    four 150M-row segments, orders 150M and customer 15M rows in one segment each (the
    reference's star join reads a dimension's first segment only). CREATE INDEX builds
    lineitem's index on orders.o_orderdate on the GPU (timed once, files written); each step
    runs the star join of lineitem with orders filtered on ten order dates, grouped by date,
    ordered by revenue, top 10. The same script over the same tables without the index runs
    as a hash join (the fused plan): both are timed and their stored rows compared."""
    import alenka_b200 as ab
    base = args.data_dir or os.path.join(tempfile.gettempdir(), "alenka_bench")
    z = sizes(args.scale)
    seg = z["orders"]
    d = os.path.join(base, f"star_s{args.scale}_seed{args.seed}")
    marker = os.path.join(d, ".complete")
    if not os.path.exists(marker):
        os.makedirs(d, exist_ok=True)
        ab.gen_three_way(d, z["customers"], z["orders"], z["lineitems"], seg, args.seed)
        with open(marker, "w") as f:
            f.write(str(z["lineitems"]))
    rows = z["lineitems"]
    setup, script, dates = star_scripts(args.seed, "bench_star.txt")
    idx = [os.path.join(d, f"lineitem.orders.o_orderdate.{g}") for g in range((rows + seg - 1) // seg)]
    sess = ab.Session(d, resident=True)
    for t in ("lineitem", "orders"):
        sess.preload(t)
    t0 = time.perf_counter()
    sess.execute(setup)
    index_s = time.perf_counter() - t0
    index_bytes = sum(os.path.getsize(p) for p in idx)
    args.warmup = max(args.warmup, 3)
    for _ in range(args.warmup):
        sess.execute(script)
    clk = clock_sampler(0)
    clk.start()
    ms, acc = timed_steps(sess, script, args.steps, torch, None)
    clocks = clk.stop()
    st = sess.stats()
    star_out = open(os.path.join(d, "bench_star.txt"), "rb").read()
    # the same script as a hash join: without the index files the star join does not apply
    for p in idx:
        os.rename(p, p + ".off")
    try:
        for _ in range(args.warmup):
            sess.execute(script)
        jms, jacc = timed_steps(sess, script, args.steps, torch, None)
        join_out = open(os.path.join(d, "bench_star.txt"), "rb").read()
    finally:
        for p in idx:
            os.rename(p + ".off", p)
    sess.close()
    peak, peak_kind = measured_peak_hbm()
    # the star join's rows: the counts of its groups (ten dates, all within the top 10)
    survivors = sum(int(ln.split(b"|")[2]) for ln in star_out.splitlines() if ln) if star_out else 0
    qb = rows * 2
    line = {
        "metric": STAR_METRIC,
        "value": rows / (ms / 1000.0), "unit": "rows/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "dtype": "int64", "data": "synthetic",
        "config": star_config(args.scale, args.seed),
        "create_index": {"seconds": index_s, "rows_per_s": rows / index_s, "index_file_bytes": index_bytes},
        "hash_join_ms_per_step": jms, "star_vs_hash_join": jms / ms,
        "hash_join_plan": {0: "operator-at-a-time", 1: "fused", 2: "fused, replayed from its CUDA graph"}.get(
            jacc["plan"], "?"),
        "verified": {"star_eq_hash_join": star_out == join_out},
        "gpu_launches": acc["kernels"],
        "query_roofline": {"bytes_per_query": qb, "bytes": "every fact row's index code at its resident width "
                           "(the survivors' gathers, a few MB, not counted)",
                           "achieved": qb / (ms / 1000.0) / 1e9, "peak": peak, "unit": "GB/s",
                           "frac": qb / (ms / 1000.0) / 1e9 / peak, "peak_source": peak_kind},
        "rows_scanned_per_step": st.rows_scanned, "star_join_rows": survivors,
        "clocks": clocks}
    if not args.no_cpu_baseline and os.path.exists(REF_BIN):
        # the reference's own star join on the host cores, a bounded sample (lineitem 60M rows)
        sc = reference_sample_scale(args.scale)
        index_s, dt, srows, sample = star_reference(os.path.join(base, "ref"), sc, args.seed, os.cpu_count() or 1,
                                                    2, 1)
        line["cpu_baseline"] = {"value": srows / dt, "unit": "rows/s", "cores": os.cpu_count() or 1,
                                "kind": "reference", "sample": sample,
                                "create_index_rows_per_s": srows / index_s}
    print(json.dumps(line), flush=True)


def run_three_way(args, torch, dist, world, rank, local):
    import alenka_b200 as ab
    base = args.data_dir or os.path.join(tempfile.gettempdir(), "alenka_bench")
    if rank == 0:
        d, fact_rows = ensure_data(base, args.scale, args.seed)
    if dist:
        dist.barrier()
    d, fact_rows = ensure_data(base, args.scale, args.seed)
    out_name = f"bench_q3_r{rank}.txt"
    script = three_way_script(args.seed, out_name)
    args.warmup = max(args.warmup, 3)

    # device-resident fused plan (value) ------------------------------------------------
    sess = ab.Session(d, resident=True, graphs=not args.no_graphs)
    for t in ("lineitem", "orders", "customer"):
        sess.preload(t)
    for _ in range(args.warmup):
        sess.execute(script)
    sess.set_timing(True)
    clk = clock_sampler(local)
    clk.start()
    ms, acc = timed_steps(sess, script, args.steps, torch, dist)
    clocks = clk.stop()
    sess.set_timing(False)
    fused_out = open(os.path.join(d, out_name), "rb").read()
    dev_ms = acc["query_dev_ms"] / args.steps
    value = fact_rows * world / (ms / 1000.0)
    plan = {0: "operator-at-a-time", 1: "fused", 2: "fused, replayed from its CUDA graph"}.get(acc["plan"], "?")

    if args.fused_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "rows/s", "ms_per_step": ms,
                              "plan": plan, "gpu_launches": acc["kernels"],
                              "device_ms_per_step": acc["query_dev_ms"] / args.steps}), flush=True)
        sess.close()
        return
    sess.close()  # each path below runs alone on the device, with its own resident copy
    # plain operator-at-a-time GPU path, resident (the baseline the fused plan is compared to)
    plain = ab.Session(d, resident=True, plain=True)
    for t in ("lineitem", "orders", "customer"):
        plain.preload(t)
    for _ in range(3):
        plain.execute(script)
    # each plain step timed alone (CUDA events on the session's stream); the median step
    # is the path's figure
    psteps = max(5, args.steps // 2)
    plain_steps = [timed_steps(plain, script, 1, torch, dist)[0] for _ in range(psteps)]
    pms = statistics.median(plain_steps)
    plain.close()
    plain_out = open(os.path.join(d, out_name), "rb").read()

    # end to end through the C ABI with host buffers ----------------------------------
    e2e_sess = ab.Session(d, resident=False)
    for _ in range(2):
        e2e_sess.execute(script)
    esteps = max(3, args.steps // 4) if fact_rows > 100_000_000 else args.steps
    ems, eacc = timed_steps(e2e_sess, script, esteps, torch, dist)
    e2e_sess.close()
    e2e_out = open(os.path.join(d, out_name), "rb").read()

    # the stored rows: every path the same, and the reference's own where it is committed
    gname, gold = golden_output(args.scale, args.seed)
    verified = {"fused_eq_plain": fused_out == plain_out, "fused_eq_e2e": fused_out == e2e_out,
                "reference_case": gname,
                "fused_eq_reference": (fused_out == gold) if gold else None}
    if not (verified["fused_eq_plain"] and verified["fused_eq_e2e"] and verified["fused_eq_reference"] in (True, None)):
        raise SystemExit(f"bench: stored rows differ: {verified}")

    peak, peak_kind = measured_peak_hbm()
    hot = None
    if acc["hot_launches"]:
        per_launch_bytes = acc["hot_bytes"] / acc["hot_launches"]
        per_launch_ms = acc["hot_ms"] / acc["hot_launches"]
        achieved = per_launch_bytes / (per_launch_ms / 1000.0) / 1e9
        hot = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
               "traffic": scaled_traffic("probe_aggregate_lineitem_three_way.md", fact_rows),
               "kernel": "probe-aggregate stage over lineitem: k_stage_vec<0, 1> (blocked streaming scan: "
                         "conjunct, orders-bitmap probe, survivor list) + k_stage_hits<false> (per-survivor "
                         "slot, aggregate inputs, warp-folded atomics), timed together",
               "algorithmic_bytes": "rows x (l_shipdate + l_orderkey stored widths) + survivors x "
                                    "(l_extendedprice + l_discount stored widths)",
               "algorithmic_bytes_per_launch": int(per_launch_bytes), "avg_launch_ms": per_launch_ms,
               "peak_source": f"{peak_kind} hbm_gbs (copy bandwidth measured on this pool)"}
    qb = query_bytes(d, fact_rows, {})
    query_roofline = {"bytes_per_query": qb, "device_ms": dev_ms, "achieved": qb / (dev_ms / 1000.0) / 1e9,
                      "peak": peak, "unit": "GB/s", "frac": qb / (dev_ms / 1000.0) / 1e9 / peak,
                      "bytes": "every referenced column of the three tables at its stored width over all rows "
                               "(no segment is skipped); the hash terms are 0: the probed bitmap fits L2",
                      "frac_wall": qb / (ms / 1000.0) / 1e9 / peak}
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(base, args.scale, args.seed, os.cpu_count() or 1)
        except Exception as e:  # test infrastructure: report, do not fail
            cpu = {"value": None, "unit": "rows/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": workload_config(args.scale, world),
            "plan": plan, "device_ms_per_step": dev_ms,
            "plain_gpu_rows_per_s": fact_rows * world / (pms / 1000.0), "fused_vs_plain": pms / ms,
            "plain_ms_steps": [round(x, 3) for x in plain_steps],
            "verified": verified,
            "e2e": {"value": fact_rows * world / (ems / 1000.0), "unit": "rows/s",
                    "h2d_bytes_per_step": eacc["h2d"] // esteps, "d2h_bytes_per_step": eacc["d2h"] // esteps},
            "gpu_launches": acc["kernels"],
            "roofline": hot,
            "query_roofline": query_roofline,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
