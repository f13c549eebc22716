#!/usr/bin/env python
"""Benchmark of the B200 InsPIRe server.

Default workload (one step = one answer batch over the whole database):
  setup(N_entries = 2^29, w = 30) -> 32768 x 262144 u16 DB (17.18 GB, 16 GiB),
  128 packing groups, 8.59 GB of precomputed tensors, one Horner chain of
  128 ciphertexts per query.  w = 30 stands in for w = 32, which the
  reference's setup() rejects; it gives the same DB byte size.  DB values:
  synthetic, splitmix64(k) mod 65535.  Queries: synthetic residues uniform in
  [0, q_l) per limb (the server's work does not depend on their values).

Reported line (rank 0): ``value`` = served q/s at batch 32, device-resident
inputs, max over ranks of the CUDA-event time of K steps; ``e2e`` = the same
through ipir_answer_batch with pinned host queries/responses (H2D + kernels +
D2H inside the timed region); plus the plain batch-1 q/s, p50/p99 latency of
the plain path, a batch sweep (B = 1, 8, 32, 64) with per-stage times, the
DB-pass GB/s, the roofline of the mat-vec kernel, the kernel schedule the
autotuner picked, the CPU baseline (the oracle port on the host cores), and
``serving``: the serving loop (cyclic scan) on the same database at 3x and
5x the plain rate, p99 over the plain p50, every response checked.

``--mode serve`` drives the continuous-batching serving loop with open-loop
Poisson arrivals over resident databases and reports p50/p95/p99 latency and
sustained q/s per offered rate, every response checked bit-exact against
the plain single answer of the same query.  ``--serve-config mixed``: a
1 GB database (setup(2^25, 30)) and a 4 GB one (setup(2^22, 960)), 70/30
split, 50/100/200/400 q/s, lane batches.  ``--serve-config 16gb``: the
default workload at 1, 3 and 5 times the plain per-query rate, cyclic scan
with 4 segments (``--serve-scan`` overrides either).

``--impl reference`` times the CPU restatement of the reference's server
path (the reference has no CPU server of its own) answering one full query
per step, unsampled, on all host threads; it loads nothing of this build.  Multi-GPU: every rank serves an independent replica.
"""
import argparse
import json
import os
import random
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "inspire-gpu_b200"))

N = 2048
Q = (94519297, 95293441)
NSTEPS = 1023
SWEEP = (1, 8, 32, 64)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="batch", choices=["batch", "serve", "matvec", "refgpu"])
    ap.add_argument("--mv-entries", type=int, default=1 << 31,
                    help="matvec mode: setup(N, 30) sizes the DB (2^31: 32768 x 1048576 u16 = 68.7 GB)")
    ap.add_argument("--mv-batches", default="1,16,32,64,128,256")
    ap.add_argument("--n-entries", type=int, default=1 << 29)
    ap.add_argument("--entry-bytes", type=int, default=30)
    ap.add_argument("--db-rows", type=int, default=0,
                    help="db_rows for setup() (0: its default); e.g. 2048 with --n-entries 8388608 --entry-bytes 120 "
                         "gives the 16 GB geometry's 128 groups on a 1 GB DB")
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the shortened runs of configurations 2 (1 GB single-query path), 5 (mixed serving, "
                         "5 s per rate) and 4 (64 GB mat-vec) that the default run appends under `configs`")
    ap.add_argument("--no-serve-check", action="store_true",
                    help="skip the serving-loop check (cyclic scan at 3x and 5x the plain rate) of the default run")
    ap.add_argument("--serve-config", default="mixed", choices=["mixed", "16gb"])
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-rates", default="")
    ap.add_argument("--query-pool", action="store_true",
                    help="serve mode: replay a pool of 32 queries per database instead of one fresh query per "
                         "request from the GPU load generator")
    ap.add_argument("--serve-lanes", type=int, default=2)
    ap.add_argument("--serve-max-batch", type=int, default=64)
    ap.add_argument("--serve-overlap", action="store_true",
                    help="admit batches while the previous DB pass of their database still runs")
    ap.add_argument("--serve-scan", type=int, default=None,
                    help="cyclic scan: DB and tensor passes as this many segments in rotation, requests join "
                         "at the next segment (databases whose columns split into multiples of 128); 0: lane "
                         "batches; -1: chosen per database from its plain answer (scan from 2 ms); default 4 "
                         "for --serve-config 16gb, 0 for mixed (the faster of each)")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def max_over_ranks(x, world, device):
    """Max of a per-rank time over all ranks (a collective: every rank calls it)."""
    if world == 1:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replicas_value(per_step_ms, batch, world):
    """Whole-job q/s of `world` replicas each answering `batch` queries per step."""
    return world * batch * 1000.0 / per_step_ms


def describe(params):
    R, C, G = params["db_rows"], params["db_cols"], params["n_packed"]
    ne, w = params["n_entries"], params["entry_bytes"]
    ne_s = f"2^{ne.bit_length() - 1}" if ne & (ne - 1) == 0 else str(ne)
    return (f"setup({ne_s}, w={w}): {R} x {C} u16 DB ({R * C * 2 / 1e9:.2f} GB), {G} groups, "
            f"{G * 2 * (2 * NSTEPS * 2 * N * 4) / 1e9:.2f} GB tensors, {params['num_cts']} ct/query")


def synth_queries(params, count, seed, out):
    """Uniform residues per limb in the flat query layout (ref src/capi.h:109-112)."""
    rng = np.random.default_rng(seed)
    R = params["db_rows"]
    blk = 2 * 2 * N
    for i in range(count):
        q = out[i]
        q[:R] = rng.integers(0, Q[0], R, dtype=np.uint64)
        q[R:2 * R] = rng.integers(0, Q[1], R, dtype=np.uint64)
        rest = q[2 * R:].reshape(-1, N)              # [.. ][digit][limb][N] blocks
        for r in range(rest.shape[0]):
            rest[r] = rng.integers(0, Q[r & 1], N, dtype=np.uint64)
        assert rest.size == 6 * blk


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML every 5 ms
    during the timed region (read-only queries)."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, cuda_index):
        self.cuda_index = cuda_index
        self.sm, self.reasons, self.max_mhz = [], set(), None
        self.err = None
        self._stop = threading.Event()
        self.t = None

    def _handle(self, nv):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.cuda_index).uuid)
            return nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            masks = [(name, getattr(nv, attr)) for name, attr in self.REASONS]

            def loop():
                while not self._stop.is_set():
                    try:
                        self.sm.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                        r = get_reasons(h)
                        for name, m in masks:
                            if r & m:
                                self.reasons.add(name)
                    except Exception as e:  # keep sampling; report the error
                        self.err = str(e)
                    self._stop.wait(0.005)

            self.t = threading.Thread(target=loop, daemon=True)
            self.t.start()
        except Exception as e:
            self.err = f"nvml unavailable: {e}"

    def stop(self):
        self._stop.set()
        if self.t is not None:
            self.t.join(timeout=5)
        d = {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.max_mhz,
             "reasons": sorted(self.reasons), "samples": len(self.sm), "source": "nvml, 5 ms"}
        if self.err:
            d["error"] = self.err
        return d


# DRAM bytes per algorithmic byte of mv_tc_kernel, from one ncu capture of a
# batch-1 launch on the 1 GB geometry (dram__bytes_read.sum 1,074,709,760 +
# dram__bytes_write.sum 5,927,168 for 1,074,266,112 algorithmic bytes); the
# kernel streams the DB once, so its traffic scales with the DB size.
MV_TC_TRAFFIC_RATIO = (1074709760 + 5927168) / 1074266112


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU leg
def host_mem_available():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return None


class CpuQuery:
    """The CPU restatement of the reference's server path (the oracle port:
    orc_answer = mat-vec over every DB column, the tensor pass of every group
    in parallel on all host threads, the full Horner chain) answering one
    whole query, unsampled.  Geometry comes from the reference's own setup()
    (its CPU library built from its sources); the DB, the precomputed
    tensors and the query are synthetic residues (the work does not depend
    on their values).  If the host cannot hold the DB and the tensors, the
    1 GB geometry setup(2^25, 30) is used instead and the sample says so."""

    def __init__(self, n_entries, w):
        sys.path.insert(0, os.path.join(REPO, "tests"))
        from oracle_lib import PRE_A, PRE_D, PRE_F, Oracle, RefLib
        self.o = Oracle()
        self.threads = self.o.L.orc_num_threads()
        ref = RefLib()
        geom = ref.setup(n_entries, w)
        need = lambda g: g[2] * g[3] * 2 + g[4] * (PRE_A + 2 * PRE_D + PRE_F) * 4
        avail = host_mem_available()
        self.note = ""
        if avail is not None and need(geom) > 0.7 * avail:
            self.note = (f"; host MemAvailable {avail / 1e9:.0f} GB cannot hold the {need(geom) / 1e9:.1f} GB "
                         f"geometry, so the 1 GB geometry setup(2^25, 30) is timed instead")
            geom = ref.setup(1 << 25, 30)
        self.geom = geom
        _, _, R, Cc, G, D, ncts = geom
        self.R, self.C, self.D = R, Cc, D
        t0 = time.perf_counter()
        self.db = self.o.fill_db(R * Cc, 0)
        self.pa = self.o.fill_u32_mod(G * PRE_A, 1, Q[0])
        self.pdp = self.o.fill_u32_mod(G * PRE_D, 2, Q[0])
        self.pdm = self.o.fill_u32_mod(G * PRE_D, 3, Q[0])
        self.pdf = self.o.fill_u32_mod(G * PRE_F, 4, Q[0])
        self.fill_s = time.perf_counter() - t0
        rng = np.random.default_rng(5)
        qn = 2 * R + 6 * 2 * 2 * N
        q = np.empty(qn, np.uint64)
        q[:R] = rng.integers(0, Q[0], R, dtype=np.uint64)
        q[R:2 * R] = rng.integers(0, Q[1], R, dtype=np.uint64)
        rest = q[2 * R:].reshape(-1, N)
        for r in range(rest.shape[0]):
            rest[r] = rng.integers(0, Q[r & 1], N, dtype=np.uint64)
        self.q = q
        self.resp = np.zeros(ncts * 4 * N, np.uint64)

    def answer_s(self):
        from oracle_lib import ptr, u16p, u32p, u64p
        args = (ptr(self.db, u16p), self.R, self.C, self.D, ptr(self.pa, u32p), ptr(self.pdp, u32p),
                ptr(self.pdm, u32p), ptr(self.pdf, u32p), ptr(self.q, u64p), ptr(self.resp, u64p))
        t0 = time.perf_counter()
        rc = self.o.L.orc_answer(*args)
        t = time.perf_counter() - t0
        assert rc == 0
        return t

    def sample(self, n_timed):
        _, _, R, Cc, G, D, ncts = self.geom
        return (f"oracle port (CPU restatement of the reference's server path), one full query per step, "
                f"unsampled and measured: mat-vec over all {R} x {Cc} DB entries, the tensor pass of all {G} "
                f"groups, {ncts} Horner chain(s) of {min(D, G) - 1} ExtProd steps; {self.threads} host threads "
                f"(OpenMP over columns and groups; the Horner chain is serial); {n_timed} timed queries; "
                f"synthetic DB, tensors and query{self.note}")


def cpu_baseline(n_entries, w, timed=2):
    """cpu_baseline of our arm's line: the same full CPU query, median of
    `timed` runs after one untimed run."""
    cq = CpuQuery(n_entries, w)
    cq.answer_s()
    ts = [cq.answer_s() for _ in range(timed)]
    t = statistics.median(ts)
    return {"value": 1.0 / t, "unit": "q/s", "cores": cq.threads, "kind": "port", "ms_per_query": t * 1e3,
            "sample": cq.sample(timed)}


def line_config(params, B, world):
    """The `config` both arms report (the same workload)."""
    db_bytes = params["db_rows"] * params["db_cols"] * 2
    return {"workload": describe(params) + f"; batch {B}",
            "server": "InsPIRe PIR server", "global_batch": B * world,
            "parallelism": f"replicas x{world}",
            "l2": f"inputs larger than L2 ({db_bytes / 1e9:.1f} GB DB read per step)"}


METRIC = "q/s at 16 GB DB (plain batch-1 vs served batch-32), p50/p99 latency, DB-pass GB/s"


# ------------------------------------------------------------------ reference arm
def run_reference(args):
    """The reference has no CPU server of its own (docs/ARCHITECTURE.md:378-380),
    so its CPU path is the oracle port: one full query per step on all host
    threads.  Nothing of this build's library is loaded here: the geometry
    comes from the reference's own setup()."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    cq = CpuQuery(args.n_entries, args.entry_bytes)
    _, _, R, Cc, G, D, ncts = cq.geom
    params = {"n_entries": cq.geom[0], "entry_bytes": cq.geom[1], "db_rows": R, "db_cols": Cc, "n_packed": G,
              "interp_d": D, "num_cts": ncts}
    for _ in range(args.warmup):
        cq.answer_s()
    ts = [cq.answer_s() for _ in range(args.steps)]
    t = sum(ts) / len(ts)
    v = 1.0 / t
    line = {"impl": "reference", "metric": METRIC,
            "value": v, "unit": "q/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64 mod q (exact, u128 dot products)", "data": "synthetic",
            "config": line_config(params, args.batch, 1),
            "queries_per_step": 1,
            "ms_per_step_p50": statistics.median(ts) * 1e3, "fill_s": cq.fill_s,
            "cpu_baseline": {"value": v, "unit": "q/s", "cores": cq.threads, "kind": "port",
                             "sample": cq.sample(args.steps)},
            "e2e": {"value": v, "unit": "q/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def serve_check(ib, srv, params, qbuf, plain_lat_ms, seconds=8.0):
    """The serving form on the benchmark's own database: a serving loop in
    cyclic-scan mode (4 segments) under open-loop Poisson arrivals at 3x and
    5x the plain per-query rate; p99 latency over the plain answer's p50,
    every response compared with the plain answer of its query."""
    pool_n = min(32, len(qbuf))
    alone = [np.stack([srv.answer(qbuf[i]) for i in range(pool_n)])]
    views = [[ib.query_view_from_flat(params, qbuf[i]) for i in range(pool_n)]]
    r1 = 1000.0 / statistics.mean(plain_lat_ms)
    p50_plain = sorted(plain_lat_ms)[len(plain_lat_ms) // 2]
    loop = ib.ServeLoop([srv], max_batch=32, queue_slots=256, scan_segments=4)
    try:
        scan = loop.db_info(0)["lanes"] == 1
        rng = random.Random(7)
        rates = []
        for x in (3, 5):
            r = serve_rate(ib, loop, [srv], PoolSource(views, alone, random.Random(8 + x)), [1.0], x * r1, seconds,
                           rng)
            rates.append({"x_plain_rate": x, "offered_q_per_s": r["offered_q_per_s"],
                          "sustained_q_per_s": r["sustained_q_per_s"], "requests": r["requests"],
                          "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"],
                          "p99_over_plain_p50": r["p99_ms"] / p50_plain if r["p99_ms"] else None,
                          "mismatches": r["mismatches"], "failed": r["failed"]})
    finally:
        loop.close()
    return {"mode": "cyclic scan, 4 segments" if scan else "lane batches", "plain_p50_ms": p50_plain,
            "plain_q_per_s": r1, "seconds_per_rate": seconds, "rates": rates,
            "bit_exact": all(r["mismatches"] == 0 and r["failed"] == 0 for r in rates)}


def serve_saturated(ib, srv, params, qbuf, seconds=3.0, outstanding=128):
    """The serving loop's capacity at batch 32: lane batches on two lanes
    (one batch's Horner chains overlap the next batch's DB pass), closed
    loop with `outstanding` requests always submitted, for `seconds`; wall
    clock, host copies included.  Every response is compared with the plain
    answer of its pool query."""
    pool_n = min(32, len(qbuf))
    alone = np.stack([srv.answer(qbuf[i]) for i in range(pool_n)])
    views = [ib.query_view_from_flat(params, qbuf[i]) for i in range(pool_n)]
    loop = ib.ServeLoop([srv], max_batch=32, lanes_per_db=2, queue_slots=outstanding + 32, scan_segments=0)
    out = np.zeros(ib.response_u64s(params), np.uint64)
    bad = done = 0
    try:
        from collections import deque
        pend = deque()
        k = 0

        def submit():
            nonlocal k
            rc, t = loop.submit_view(0, views[k % pool_n])
            assert rc == 0, (rc, ib.last_error())
            pend.append((t, k % pool_n))
            k += 1

        for _ in range(outstanding):
            submit()
        t0 = time.perf_counter()
        s0 = loop.stats()
        while time.perf_counter() - t0 < seconds:
            t, qi = pend.popleft()
            loop.wait(t, out=out)
            bad += not np.array_equal(out, alone[qi])
            done += 1
            submit()
        wall = time.perf_counter() - t0
        s1 = loop.stats()
        while pend:
            t, qi = pend.popleft()
            loop.wait(t, out=out)
            bad += not np.array_equal(out, alone[qi])
        info = loop.db_info(0)
    finally:
        loop.close()
    nb = s1["batches"] - s0["batches"]
    return {"mode": "lane batches, 2 lanes, max_batch 32, closed loop", "outstanding": outstanding,
            "seconds": seconds, "q_per_s": done / wall, "requests": done,
            "mean_batch": (s1["batched_queries"] - s0["batched_queries"]) / max(1, nb),
            "lanes": info["lanes"], "mismatches": bad, "bit_exact": bad == 0,
            "timing": "wall clock over the loop's responses, host copies included (not CUDA events)"}


def run_ours(args):
    import torch
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    import inspire_b200 as ib
    B = args.batch
    sweep = [] if args.no_sweep else [b for b in SWEEP if b != B]
    max_b = max([B] + sweep)
    params = ib.setup(args.n_entries, args.entry_bytes, args.db_rows)
    R, Ccols, G = params["db_rows"], params["db_cols"], params["n_packed"]
    db = ib.fill_db(R * Ccols, 0)
    seed = bytes(range(64))
    t0 = time.perf_counter()
    srv = ib.Server(args.n_entries, args.entry_bytes, db, db_rows=args.db_rows, max_batch=max_b, crs_seed=seed)
    t_pre = time.perf_counter() - t0
    del db
    t_tune = 0.0
    if not args.no_autotune:
        t0 = time.perf_counter()
        srv.autotune()
        t_tune = time.perf_counter() - t0
    # A dedicated stream: the handle of torch's default stream is 0, which the
    # C ABI reads as "the server's own stream".
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    srv.set_stream(stream.cuda_stream)
    qn = ib.query_u64s(params)
    rn = ib.response_u64s(params)
    qbuf_t = torch.empty((max_b, qn), dtype=torch.int64, pin_memory=True)
    qbuf = qbuf_t.numpy().view(np.uint64)
    synth_queries(params, max_b, 1000 + rank, qbuf)
    obuf_t = torch.empty((max_b, rn), dtype=torch.int64, pin_memory=True)
    obuf = obuf_t.numpy().view(np.uint64)
    views = (ib.IpirQueryView * max_b)()
    for i in range(max_b):
        views[i] = ib.query_view_from_flat(params, qbuf[i])

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def ranks_max(x):
        return max_over_ranks(x, world, "cuda")

    def device_time(count, steps, sampler=None):
        srv.stage_views(views, count)
        for _ in range(args.warmup):
            srv.run(count)
        barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
            torch.cuda.nvtx.range_push("timed")   # the headline region, for ncu --nvtx-include timed/
        n0 = srv.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            srv.run(count)
        e1.record(stream)
        while not e1.query():      # sleep-polling releases the GIL for the clock sampler thread
            time.sleep(0.0002)
        torch.cuda.synchronize()
        if sampler:
            torch.cuda.nvtx.range_pop()
        launches = srv.launch_count() - n0
        clocks = sampler.stop() if sampler else None
        barrier()
        return ranks_max(e0.elapsed_time(e1) / steps), launches, clocks

    def stage_ms(count, reps):
        srv.enable_stage_timing(True)
        srv.stage_views(views, count)
        st = []
        for _ in range(reps):
            srv.run(count)
            srv.fetch(count, obuf[:count])
            st.append(srv.stage_times())
        srv.enable_stage_timing(False)
        return {k: statistics.median(s[k] for s in st) for k in st[0]}

    st1 = stage_ms(1, max(3, args.warmup))
    stB = stage_ms(B, 3)
    ms1, _, _ = device_time(1, args.steps)
    msB, launches, clocks = device_time(B, args.steps, ClockSampler(local_rank))
    value = replicas_value(msB, B, world)
    sweep_out = {}
    for b in sorted(set(sweep + [1, B])):
        if b == B:
            ms = msB
        elif b == 1:
            ms = ms1
        else:
            ms, _, _ = device_time(b, max(3, args.steps // 2))
        sweep_out[str(b)] = {"ms_per_batch": ms, "q_per_s": b * 1000.0 / ms,
                             "stage_ms": st1 if b == 1 else (stB if b == B else stage_ms(b, 2)),
                             "schedule": srv.schedule(b)}

    # e2e through the C ABI with pinned host buffers (H2D + kernels + D2H)
    for _ in range(args.warmup):
        srv.answer_batch_rc(views, B, obuf)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rc = srv.answer_batch_rc(views, B, obuf)
        assert rc == 0, ib.last_error()
    t_e2e = ranks_max((time.perf_counter() - t0) / args.steps)
    e2e_qps = world * B / t_e2e
    # e2e with the client library's wire formats: packed queries in (unpacked
    # on the device), compressed responses out
    qb, rb, cb = srv.wire_sizes()
    wq_t = torch.empty(B * qb, dtype=torch.uint8, pin_memory=True)
    wq = wq_t.numpy()
    wq[:] = np.random.default_rng(2000 + rank).integers(0, 256, wq.size, dtype=np.uint8)
    wo_t = torch.empty((B, cb), dtype=torch.uint8, pin_memory=True)
    wo = wo_t.numpy()
    for _ in range(args.warmup):
        srv.answer_wire(wq, B, ib.RESP_COMPRESSED, out=wo)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        srv.answer_wire(wq, B, ib.RESP_COMPRESSED, out=wo)
    t_wire = ranks_max((time.perf_counter() - t0) / args.steps)
    # plain path latency distribution (one query per call, e2e)
    lat = []
    for _ in range(max(args.steps, 20)):
        t0 = time.perf_counter()
        srv.answer_batch_rc(views, 1, obuf)
        lat.append((time.perf_counter() - t0) * 1000.0)
    lat.sort()
    p50 = lat[len(lat) // 2]
    p99 = lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))]
    serving = None
    if rank == 0 and world == 1 and not args.no_serve_check:
        serving = serve_check(ib, srv, params, qbuf, lat)
        serving["saturated"] = serve_saturated(ib, srv, params, qbuf)

    mv1 = st1["matvec"]
    db_bytes = R * Ccols * 2
    alg_bytes = db_bytes + 2 * R * 8          # DB + one query's b vector per launch
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (mv1 * 1e-3) / 1e9
    tensor_bytes = G * 2 * (2 * NSTEPS * 2 * N * 4)
    sched1 = srv.schedule(1)

    line = {
        "metric": METRIC,
        "value": value, "unit": "q/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": msB, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 mod q (exact: int8 limb MMAs with s32 accumulation, u64 reductions)", "data": "synthetic",
        "config": line_config(params, B, world),
        "plain_b1": {"q_per_s": 1000.0 / ms1, "ms": ms1, "p50_ms_e2e": p50, "p99_ms_e2e": p99},
        "served": {"batch": B, "ms_per_batch": msB, "q_per_s": value / world},
        "batch_sweep": sweep_out,
        "db_pass_gbs": db_bytes / (mv1 * 1e-3) / 1e9,
        "stage_ms_b1": st1, "stage_ms_batch": stB,
        "preprocess_s": t_pre, "autotune_s": t_tune,
        "roofline": {"kernel": ("mv_tc_kernel (tcgen05 int8 DB pass, batch 1)" if sched1["matvec_tc"]
                                else "matvec_kernel<1,8> (CUDA-core DB pass, batch 1)"), "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind,
                     "traffic": alg_bytes * MV_TC_TRAFFIC_RATIO if sched1["matvec_tc"] else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch on the 1 GB "
                                       "geometry, scaled by the DB size",
                     "alg_bytes_per_launch": alg_bytes},
        "tensor_pass_gbs_b1": tensor_bytes / (st1["collapse"] * 1e-3) / 1e9,
        "e2e": {"value": e2e_qps, "unit": "q/s", "h2d_bytes_per_step": B * qn * 8,
                "d2h_bytes_per_step": B * rn * 8},
        "e2e_wire": {"value": world * B / t_wire, "unit": "q/s", "h2d_bytes_per_step": B * qb,
                     "d2h_bytes_per_step": B * cb,
                     "formats": "packed queries (53-bit), compressed responses (28/20-bit)"},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if serving:
        line["serving"] = serving
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.n_entries, args.entry_bytes)
    srv.close()
    if rank == 0 and world == 1 and not args.no_configs:
        # the other configurations, shortened, so one default run records them all
        import argparse as _ap
        a5 = _ap.Namespace(**vars(args))
        a5.serve_config, a5.serve_seconds, a5.serve_rates, a5.serve_scan = "mixed", 5.0, "", None
        a5.query_pool, a5.no_autotune, a5.serve_max_batch, a5.serve_lanes, a5.serve_overlap = False, False, 64, 2, False
        line["configs"] = {
            "config2_1gb_single_query": config2(ib),
            "config5_mixed_serving_5s_per_rate": serve_sweep(a5),
            "config4_matvec_64gb": matvec_sweep(1 << 31, [1, 16, 32, 64, 128, 256], cuda_core_max_b=16, quick=True),
        }
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ serving loop
class PoolSource:
    """Requests drawn from a pool of queries per database; every response is
    compared with the plain answer of its pool query (alone[db][index])."""

    def __init__(self, views, alone, rng):
        self.views, self.alone, self.rng = views, alone, rng

    def pick(self, k):
        qi = self.rng.randrange(len(self.views[k]))
        return qi, self.views[k][qi]

    def verify(self, k, key, out):
        return np.array_equal(out, self.alone[k][key])


class FreshSource:
    """One fresh synthetic query per request from the GPU load generator
    (ipir_b200_synth_queries): a producer thread per database generates
    chunks of queries on a side stream and copies them into pinned host
    buffers, which the submitter hands to the serving loop (it copies each
    request at submit).  Each response's 64-bit hash is recorded; check()
    later regenerates every request's query from its id, answers it through
    the blocking answer of the same database handle (batches of up to 32,
    bit-identical to single answers) and compares hashes."""
    CH = 32

    def __init__(self, ib, servers, seed):
        import queue
        import torch
        self.ib, self.servers, self.seed = ib, servers, seed
        self.qn = [ib.query_u64s(s.params) for s in servers]
        self.next_id = [0] * len(servers)
        self.ready = [queue.Queue(maxsize=2) for _ in servers]
        self.free = [queue.Queue() for _ in servers]
        self.dev = [torch.empty((self.CH, q), dtype=torch.int64, device="cuda") for q in self.qn]
        for k, q in enumerate(self.qn):
            for _ in range(3):
                self.free[k].put(torch.empty((self.CH, q), dtype=torch.int64, pin_memory=True))
        self.cur = [None] * len(servers)
        rng = np.random.default_rng(seed)
        self.W = [rng.integers(0, 2 ** 63, ib.response_u64s(s.params), dtype=np.uint64) | np.uint64(1)
                  for s in servers]
        self.tag = 0                 # the offered rate the requests belong to
        self.hashes = {}             # (db, id) -> (tag, hash)
        self.stop = False
        self.device = torch.cuda.current_device()
        self.threads = [threading.Thread(target=self._produce, args=(k,), daemon=True) for k in range(len(servers))]
        for t in self.threads:
            t.start()

    def _gen(self, k, first, n, host, stream):
        self.ib.synth_queries_device(self.servers[k].params["db_rows"], self.seed + k, first, n,
                                     self.dev[k].data_ptr(), stream.cuda_stream)
        host[:n].copy_(self.dev[k][:n], non_blocking=True)
        stream.synchronize()

    def _produce(self, k):
        import queue
        import torch
        torch.cuda.set_device(self.device)
        stream = torch.cuda.Stream()
        first = 0
        while not self.stop:
            try:
                buf = self.free[k].get(timeout=0.1)
            except queue.Empty:
                continue
            with torch.cuda.stream(stream):
                self._gen(k, first, self.CH, buf, stream)
            self.ready[k].put((first, buf))
            first += self.CH

    def pick(self, k):
        c = self.cur[k]
        if c is None or c[2] == self.CH:
            if c is not None:
                self.free[k].put(c[1])
            first, buf = self.ready[k].get()
            arr = buf.numpy().view(np.uint64)
            c = self.cur[k] = [first, buf, 0, arr]
        i = c[2]
        c[2] += 1
        qid = c[0] + i
        return qid, self.ib.query_view_from_flat(self.servers[k].params, c[3][i])

    def _hash(self, k, out):
        with np.errstate(over="ignore"):
            return int((out.view(np.uint64) * self.W[k]).sum(dtype=np.uint64))

    def verify(self, k, key, out):
        self.hashes[(k, key)] = (self.tag, self._hash(k, out))
        return None

    def close(self):
        self.stop = True
        for t in self.threads:
            t.join(timeout=5)

    def check(self):
        """Mismatches and checked requests per tag."""
        import torch
        bad, checked = {}, {}
        stream = torch.cuda.Stream()
        host = torch.empty((self.CH, max(self.qn)), dtype=torch.int64, pin_memory=True)
        for k, srv in enumerate(self.servers):
            ids = sorted(i for (kk, i) in self.hashes if kk == k)
            out = np.zeros((self.CH, self.ib.response_u64s(srv.params)), np.uint64)
            pos = 0
            while pos < len(ids):
                first = ids[pos] - ids[pos] % self.CH
                chunk = [i for i in ids[pos:pos + self.CH] if i < first + self.CH]
                hbuf = host[:, :self.qn[k]]
                with torch.cuda.stream(stream):
                    self._gen(k, first, self.CH, hbuf, stream)
                arr = hbuf.numpy().view(np.uint64)
                got = srv.answer_batch([arr[i - first] for i in chunk], out=out[:len(chunk)])
                for j, i in enumerate(chunk):
                    tag, h = self.hashes[(k, i)]
                    checked[tag] = checked.get(tag, 0) + 1
                    if self._hash(k, got[j]) != h:
                        bad[tag] = bad.get(tag, 0) + 1
                pos += len(chunk)
        return bad, checked


def serve_rate(ib, loop, servers, source, split, rate, seconds, rng):
    """Open-loop Poisson arrivals at `rate` q/s for `seconds` on a serving
    loop; every response is checked by `source.verify` (a pool query against
    its plain answer, or a fresh query's hash recorded for a later check)."""
    s0 = loop.stats()
    tickets = []          # (ticket, db, pool index)
    lock = threading.Lock()
    done = {"lat": [], "queue": [], "slow": [], "bad": 0, "n": 0, "failed": 0}
    t_start = time.perf_counter()
    finished = threading.Event()

    def collector():
        outs = [np.zeros(ib.response_u64s(s.params), np.uint64) for s in servers]
        i = 0
        while True:
            with lock:
                item = tickets[i] if i < len(tickets) else None
            if item is None:
                if finished.is_set():
                    with lock:
                        if i >= len(tickets):
                            return
                    continue
                time.sleep(0.0002)
                continue
            t, k, qi, t_arr = item
            lq = C_wait(loop, t, outs[k])
            if lq is None:
                done["failed"] += 1
            else:
                done["lat"].append(lq[0])
                done["queue"].append(lq[1])
                if lq[0] > 10.0:
                    done["slow"].append((round(t_arr - t_start, 3), round(lq[0], 2), round(lq[1], 2), k))
                if source.verify(k, qi, outs[k]) is False:
                    done["bad"] += 1
            done["n"] += 1
            i += 1

    th = threading.Thread(target=collector)
    th.start()
    t_next = t_start
    full = 0
    late = 0.0
    while True:
        t_next += rng.expovariate(rate)
        if t_next - t_start > seconds:
            break
        while True:
            d = t_next - time.perf_counter()
            if d <= 0:
                break
            time.sleep(min(d, 0.001) if d > 0.0015 else 0)
        k = 0 if rng.random() < split[0] else 1 if len(servers) > 1 else 0
        qi, view = source.pick(k)
        while True:
            rc, t = loop.submit_view(k, view)
            if rc != ib.SERVE_FULL:
                break
            full += 1
            time.sleep(0.0005)
        assert rc == 0, (rc, ib.last_error())
        late = max(late, time.perf_counter() - t_next)
        with lock:
            tickets.append((t, k, qi, t_next))
    finished.set()
    th.join()
    wall = time.perf_counter() - t_start
    s1 = loop.stats()
    lat = sorted(done["lat"])

    def pct(p):
        return lat[min(len(lat) - 1, int(round(p * (len(lat) - 1))))] if lat else None

    qs = sorted(done["queue"])

    def qpct(p):
        return qs[min(len(qs) - 1, int(round(p * (len(qs) - 1))))] if qs else None

    tr = [r for r in loop.trace() if r["t_issue_s"] >= t_start]
    slow_batches = sorted(([round(r["t_issue_s"] - t_start, 3), round(r["issue_ms"], 2), round(r["device_ms"], 2),
                            round(r["notice_ms"], 3), r["db"], r["lane"], r["count"]]
                           for r in tr if r["device_ms"] > 5.0 or r["issue_ms"] > 2.0), key=lambda x: x[0])
    dev = sorted(r["device_ms"] for r in tr)
    nb = s1["batches"] - s0["batches"]
    return {"offered_q_per_s": rate, "sustained_q_per_s": done["n"] / wall,
            "requests": done["n"], "p50_ms": pct(0.50), "p95_ms": pct(0.95), "p99_ms": pct(0.99),
            "max_ms": lat[-1] if lat else None, "mismatches": done["bad"], "failed": done["failed"],
            "batches": nb, "mean_batch": (s1["batched_queries"] - s0["batched_queries"]) / max(1, nb),
            "queue_full_retries": full, "queue_p50_ms": qpct(0.5), "queue_p99_ms": qpct(0.99),
            "slow_over_10ms": done["slow"][:20], "max_notice_ms": s1["max_notice_ms"],
            "batch_device_ms_p50": dev[len(dev) // 2] if dev else None,
            "batch_device_ms_max": dev[-1] if dev else None,
            "slow_batches_t_issue_dev_notice_db_lane_n": slow_batches[:20],
            "generator_max_late_ms": late * 1e3}


def run_serve(args):
    """Open-loop Poisson load on the continuous-batching serving loop."""
    print(json.dumps(serve_sweep(args)), flush=True)


def serve_sweep(args):
    """The serving loop under open-loop Poisson arrivals at each offered rate
    (configuration 5 with --serve-config mixed); returns the JSON object."""
    import torch
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    import inspire_b200 as ib
    if args.serve_config == "mixed":
        dbs = [(1 << 25, 30, 0, bytes([7] * 64)), (1 << 22, 960, 1, bytes([9] * 64))]
        split = [0.7, 0.3]
        rates = [50.0, 100.0, 200.0, 400.0]
    else:
        dbs = [(args.n_entries, args.entry_bytes, 0, bytes(range(64)))]
        split = [1.0]
        rates = None   # multiples of the plain rate, below
    servers, pools, alone, plain = [], [], [], []
    pool_n = 32
    for k, (ne, w, dseed, cseed) in enumerate(dbs):
        p = ib.setup(ne, w)
        db = ib.fill_db(p["db_rows"] * p["db_cols"], dseed)
        srv = ib.Server(ne, w, db, max_batch=32, crs_seed=cseed)
        del db
        servers.append(srv)
        qs = np.zeros((pool_n, ib.query_u64s(p)), np.uint64)
        synth_queries(p, pool_n, 100 + k, qs)
        pools.append(qs)
        alone.append(np.stack([srv.answer(q) for q in qs]))
        lat = []
        for i in range(30):
            t0 = time.perf_counter()
            srv.answer(qs[i % pool_n])
            lat.append((time.perf_counter() - t0) * 1e3)
        lat.sort()
        plain.append({"workload": describe(p), "p50_ms": lat[len(lat) // 2], "p99_ms": lat[-1],
                      "q_per_s": 1e3 / statistics.mean(lat)})
    if rates is None:
        r1 = plain[0]["q_per_s"]
        rates = [r1, 3 * r1, 5 * r1]
    if args.serve_scan is None:
        args.serve_scan = 4 if args.serve_config == "16gb" else 0
    if args.serve_rates:
        rates = [float(x) for x in args.serve_rates.split(",")]
    t0 = time.perf_counter()
    loop = ib.ServeLoop(servers, max_batch=args.serve_max_batch, lanes_per_db=args.serve_lanes, queue_slots=512,
                        overlap_db_passes=args.serve_overlap, scan_segments=args.serve_scan,
                        autotune=not args.no_autotune)
    t_create = time.perf_counter() - t0
    views = [[ib.query_view_from_flat(servers[k].params, pools[k][i]) for i in range(pool_n)]
             for k in range(len(dbs))]
    results = []
    rng = random.Random(6)
    source = PoolSource(views, alone, random.Random(7)) if args.query_pool else FreshSource(ib, servers, 6000)
    for tag, rate in enumerate(rates):
        source.tag = tag
        results.append(serve_rate(ib, loop, servers, source, split, rate, args.serve_seconds, rng))
    infos = [loop.db_info(k) for k in range(len(dbs))]
    loop.close()
    if not args.query_pool:
        source.close()
        t0 = time.perf_counter()
        bad, checked = source.check()
        for tag, r in enumerate(results):
            r["mismatches"] = bad.get(tag, 0)
            r["checked"] = checked.get(tag, 0)
        t_check = time.perf_counter() - t0
    else:
        t_check = 0.0
    for s in servers:
        s.close()
    line = {"metric": "serving loop: p50/p95/p99 latency and sustained q/s under open-loop Poisson arrivals",
            "mode": "serve", "config": {"workload": args.serve_config, "databases": [p["workload"] for p in plain],
                                        "split": split, "seconds_per_rate": args.serve_seconds,
                                        "max_batch": args.serve_max_batch, "lanes_per_db": args.serve_lanes,
                                        "overlap_db_passes": args.serve_overlap,
                                        "scan_segments": args.serve_scan, "autotune": not args.no_autotune},
            "n_gpus": 1, "unit": "ms",
            "data": ("synthetic queries (pool of 32 per database)" if args.query_pool else
                     "fresh synthetic queries from the GPU load generator (ipir_b200_synth_queries), one per "
                     "request; every response checked afterwards against the blocking answer of its regenerated "
                     "query by 64-bit hash"),
            "plain": plain, "rates": results, "create_s": t_create, "check_s": t_check,
            "lanes": [{"lanes": i["lanes"], "max_batch": i["max_batch"]} for i in infos],
            "bit_exact_vs_alone": all(r["mismatches"] == 0 and r["failed"] == 0 for r in results)}
    return line


def config2(ib, n_queries=256):
    """Configuration 2, the single-query path at 1 GB: setup(2^25, 30), DB
    from seed 0, gpu_preprocess timed (ipir_server_create from the host DB),
    then n_queries sequential plain answers through ipir_answer_batch (fresh
    synthetic queries from the GPU load generator, seed 3), and the batch-1
    DB pass in GB/s from the stage timers.  Bit-exactness at this geometry
    against the reference's own GPU build is the parity test
    tests/test_gpu_vs_reference_gpu_geoms.py (cfg2)."""
    import torch
    p = ib.setup(1 << 25, 30)
    R, Cc = p["db_rows"], p["db_cols"]
    db = ib.fill_db(R * Cc, 0)
    t0 = time.perf_counter()
    srv = ib.Server(1 << 25, 30, db, max_batch=1, crs_seed=bytes([1] * 64))
    t_pre = time.perf_counter() - t0
    del db
    qn = ib.query_u64s(p)
    dq = torch.empty((n_queries, qn), dtype=torch.int64, device="cuda")
    ib.synth_queries_device(R, 3, 0, n_queries, dq.data_ptr())
    hq = dq.cpu().numpy().view(np.uint64)
    del dq
    out = np.zeros(ib.response_u64s(p), np.uint64)
    views = (ib.IpirQueryView * n_queries)()
    for i in range(n_queries):
        views[i] = ib.query_view_from_flat(p, hq[i])
    for i in range(3):
        srv.answer_batch_rc(views, 1, out)
    lat = []
    for i in range(n_queries):
        t1 = time.perf_counter()
        rc = srv.answer_batch_rc(C_view(views, i), 1, out)
        lat.append((time.perf_counter() - t1) * 1e3)
        assert rc == 0
    srv.enable_stage_timing(True)
    st = []
    for i in range(5):
        srv.answer_batch_rc(C_view(views, i), 1, out)
        st.append(srv.stage_times())
    srv.enable_stage_timing(False)
    srv.close()
    stm = {k: statistics.median(x[k] for x in st) for k in st[0]}
    peak, kind = measured_peaks()
    lat.sort()
    gbs = R * Cc * 2 / (stm["matvec"] * 1e-3) / 1e9
    return {"workload": describe(p), "preprocess_s": t_pre, "answers": n_queries,
            "p50_ms_e2e": lat[len(lat) // 2], "p99_ms_e2e": lat[min(len(lat) - 1, int(0.99 * (len(lat) - 1)))],
            "q_per_s_e2e": n_queries * 1e3 / sum(lat), "stage_ms_b1": stm, "db_pass_gbs": gbs,
            "db_pass_frac": gbs / peak, "peak_source": kind,
            "parity": "bit-exact vs the reference GPU build at this geometry: tests/test_gpu_vs_reference_gpu_geoms.py"}


def C_view(views, i):
    """The query view array starting at element i (ctypes pointer arithmetic)."""
    import ctypes as C
    return C.cast(C.addressof(views) + i * C.sizeof(views._type_), C.POINTER(views._type_))


def splitmix_mod(idx, seed):
    """Host copy of the synthetic DB formula on an index array (u64)."""
    with np.errstate(over="ignore"):
        x = (idx ^ np.uint64(seed)) + np.uint64(0x9e3779b97f4a7c15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
        x ^= x >> np.uint64(31)
    return x % np.uint64(65535)


def run_matvec(args):
    import torch
    torch.cuda.set_device(0)
    print(json.dumps(matvec_sweep(args.mv_entries, [int(x) for x in args.mv_batches.split(",")])), flush=True)


def matvec_sweep(mv_entries, Bs, cuda_core_max_b=None, quick=False):
    """Exact mat-vec microbench (configuration 4): DB x B queries on the
    tensor cores and on the CUDA cores, each B's schedule autotuned (quick:
    the default schedule only), sampled columns checked against exact host
    dot products.  Returns the JSON object."""
    import torch
    import inspire_b200 as ib
    params = ib.setup(mv_entries, 30)
    R, Cc = params["db_rows"], params["db_cols"]
    db_seed, q_seed = 0, 5
    db = torch.empty(R * Cc, dtype=torch.int16, device="cuda")
    ib.fill_db_device(db.data_ptr(), R * Cc, db_seed)
    Bmax = max(Bs)
    rng = np.random.default_rng(q_seed)
    qh = np.empty((Bmax, 2, R), np.uint64)
    qh[:, 0, :] = rng.integers(0, Q[0], (Bmax, R), dtype=np.uint64)
    qh[:, 1, :] = rng.integers(0, Q[1], (Bmax, R), dtype=np.uint64)
    q = torch.from_numpy(qh.view(np.int64).reshape(-1)).cuda()
    out = torch.empty(Bmax * 2 * Cc, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    db_bytes = R * Cc * 2
    hbm_peak, peak_kind = measured_peaks()
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            int8_peak = 2 * float(json.load(f)["bf16_tflops"])   # dense int8 = 2x dense bf16 (4.5 vs 2.25 P nominal)
        int8_kind = "2 x measured bf16 GEMM"
    except Exception:
        int8_peak, int8_kind = 4500.0, "nominal"
    # sampled columns for the exact check (the host regenerates them)
    cs = np.sort(np.random.default_rng(1).choice(Cc, 24, replace=False)).astype(np.uint64)
    rows_idx = np.arange(R, dtype=np.uint64)[:, None] * np.uint64(Cc)
    dcols = splitmix_mod(rows_idx + cs[None, :], db_seed)          # (R, 24) u64, < 2^16

    def timed(B, path, qpp, kc, reps):
        ib.matvec_ex(db.data_ptr(), R, Cc, q.data_ptr(), B, out.data_ptr(), path, qpp, kc, sh, True)  # warm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            ib.matvec_ex(db.data_ptr(), R, Cc, q.data_ptr(), B, out.data_ptr(), path, qpp, kc, sh, False)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def check(B):
        oh = out[:B * 2 * Cc].cpu().numpy().view(np.uint32).reshape(B, 2, Cc)
        bad = 0
        for l, mod in enumerate(Q):
            exp = (qh[:B, l, :] @ dcols) % np.uint64(mod)             # exact: sums < 2^59
            bad += int((oh[:, l, cs.astype(np.int64)].astype(np.uint64) != exp).sum())
        return bad

    results = {}
    for B in Bs:
        row = {}
        for path in (0, 1):
            if path == 1 and cuda_core_max_b is not None and B > cuda_core_max_b:
                continue
            if path == 0 and not quick:
                qpps = sorted({min(B, 32)} | ({16, 8} if B > 16 else set()) | ({B} if B < 32 else set()))
                kcs = [0] + [k for k in (8192, 16384) if R % k == 0 and k < R]
            elif path == 0:
                qpps, kcs = [min(B, 32)], [0]
            else:
                qpps, kcs = [min(B, 4)], [0]
            best = None
            for qpp in qpps:
                for kc in kcs:
                    passes = -(-B // qpp)
                    reps = max(1, min(5, int(4000 / (passes * (12 if path == 0 else 60)))))
                    ms = timed(B, path, qpp, kc, reps)
                    if best is None or ms < best[0]:
                        best = (ms, qpp, kc)
            ms, qpp, kc = best
            ib.matvec_ex(db.data_ptr(), R, Cc, q.data_ptr(), B, out.data_ptr(), path, qpp, kc, sh, True)
            torch.cuda.synchronize()
            passes = -(-B // qpp)
            ops = 2 * 14 * B * R * Cc           # 7 CRT query planes x 2 DB bytes per (row, col), 2 ops per MAC
            d = {"ms": ms, "q_per_s": B * 1e3 / ms, "db_passes": passes,
                 "hbm_gbs": passes * db_bytes / (ms * 1e-3) / 1e9,
                 "hbm_frac": passes * db_bytes / (ms * 1e-3) / 1e9 / hbm_peak,
                 "schedule": {"queries_per_pass": qpp, "kchunk_rows": kc or "auto"},
                 "sampled_mismatches": check(B)}
            if path == 0:
                d["int8_tops"] = ops / (ms * 1e-3) / 1e12
                d["int8_frac"] = d["int8_tops"] / int8_peak
            row["tensor_cores" if path == 0 else "cuda_cores"] = d
        results[str(B)] = row
    del db, q, out
    torch.cuda.empty_cache()
    return {"metric": "exact mat-vec microbench: ms, q/s, HBM GB/s and int8 TOPS per batch (tensor vs CUDA cores)",
            "mode": "matvec", "n_gpus": 1, "data": "synthetic",
            "config": {"workload": f"setup(2^{mv_entries.bit_length() - 1}, w=30): {R} x {Cc} u16 DB "
                                   f"({db_bytes / 1e9:.1f} GB, splitmix64 seed {db_seed}), queries uniform in [0, q) "
                                   f"per limb (seed {q_seed})",
                       "check": "24 sampled columns x all queries x both limbs vs exact host dot products"},
            "peaks": {"hbm_gbs": hbm_peak, "hbm_source": peak_kind, "int8_tops": int8_peak, "int8_source": int8_kind},
            "results": results,
            "bit_exact": all(v[p]["sampled_mismatches"] == 0 for v in results.values() for p in v)}


def run_refgpu(args):
    """The reference's own GPU server library (compiled for sm_100a from its
    sources into oracle/_ref by oracle/Makefile) on the same workload,
    through its own C ABI: preprocess time, plain batch-1 latency and
    batch-B q/s from host buffers (its ipir_answer_batch copies queries in
    and responses out, like our e2e)."""
    import ctypes as C
    path = os.path.join(REPO, "oracle", "_ref", "libinspire_ref_gpu.so")
    if not os.path.exists(path):
        print(json.dumps({"impl": "reference_gpu", "unavailable": "oracle/_ref/libinspire_ref_gpu.so not built"}))
        return
    import inspire_b200 as ib
    R_ = C.CDLL(path)  # RTLD_LOCAL: its ipir_* names do not interpose on ours
    R_.ipir_server_create.restype = C.c_void_p
    R_.ipir_server_create.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p,
                                      C.POINTER(ib.IpirParams)]
    R_.ipir_answer_batch.argtypes = [C.c_void_p, C.POINTER(ib.IpirQueryView), C.c_size_t, C.c_void_p]
    R_.ipir_server_destroy.argtypes = [C.c_void_p]
    B = args.batch
    params = ib.setup(args.n_entries, args.entry_bytes)
    R, Cc = params["db_rows"], params["db_cols"]
    db = ib.fill_db(R * Cc, 0)
    seed = np.frombuffer(bytes(range(64)), np.uint8).copy()
    p = ib.IpirParams()
    t0 = time.perf_counter()
    h = R_.ipir_server_create(args.n_entries, args.entry_bytes, 0, B, db.ctypes.data, seed.ctypes.data, C.byref(p))
    t_pre = time.perf_counter() - t0
    del db
    if not h:
        print(json.dumps({"impl": "reference_gpu", "unavailable": "ipir_server_create failed"}))
        return
    qn, rn = ib.query_u64s(params), ib.response_u64s(params)
    qbuf = np.zeros((B, qn), np.uint64)
    synth_queries(params, B, 1000, qbuf)
    obuf = np.zeros((B, rn), np.uint64)
    views = (ib.IpirQueryView * B)()
    for i in range(B):
        views[i] = ib.query_view_from_flat(params, qbuf[i])
    for _ in range(args.warmup):
        assert R_.ipir_answer_batch(h, views, 1, obuf.ctypes.data) == 0
    lat = []
    for _ in range(max(args.steps, 20)):
        t0 = time.perf_counter()
        R_.ipir_answer_batch(h, views, 1, obuf.ctypes.data)
        lat.append((time.perf_counter() - t0) * 1e3)
    lat.sort()
    for _ in range(args.warmup):
        R_.ipir_answer_batch(h, views, B, obuf.ctypes.data)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        assert R_.ipir_answer_batch(h, views, B, obuf.ctypes.data) == 0
    t_b = (time.perf_counter() - t0) / args.steps
    R_.ipir_server_destroy(h)
    print(json.dumps({"impl": "reference_gpu", "metric": "reference GPU server on this B200: preprocess s, plain "
                      "latency, batch q/s (host buffers)", "config": {"workload": describe(params), "batch": B},
                      "preprocess_s": t_pre, "plain_p50_ms": lat[len(lat) // 2], "plain_p99_ms": lat[-1],
                      "batch_ms": t_b * 1e3, "batch_q_per_s": B / t_b,
                      "build": "oracle/Makefile ref_gpu: its five .cu files + CPU sources, nvcc sm_100a -O3"}),
          flush=True)


def C_wait(loop, ticket, out):
    import inspire_b200 as ib
    try:
        return loop.wait(ticket, out=out, timeout=120.0, with_queue=True)
    except ib.InspireError:
        return None


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "serve":
        rank, _, _ = dist_env()
        if rank == 0:
            run_serve(args)
    elif args.mode == "matvec":
        rank, _, _ = dist_env()
        if rank == 0:
            run_matvec(args)
    elif args.mode == "refgpu":
        rank, _, _ = dist_env()
        if rank == 0:
            run_refgpu(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
