#!/usr/bin/env python
"""Benchmark of the B200 InsPIRe server on the 16 GB configuration.

Workload (one step = one answer batch over the whole database):
  setup(N_entries = 2^29, w = 30) -> 32768 x 262144 u16 DB (17.18 GB, 16 GiB),
  128 packing groups, 8.59 GB of precomputed tensors, one Horner chain of
  128 ciphertexts per query.  w = 30 stands in for the configuration's w = 32,
  which the reference's setup() rejects; it gives the same DB byte size.
  DB values: synthetic, splitmix64(k) mod 65535.  Queries: synthetic residues
  uniform in [0, q_l) per limb (the server's work does not depend on them).

Reported line (rank 0): ``value`` = served q/s at batch 32, device-resident
inputs, max over ranks of the CUDA-event time of K steps; ``e2e`` = the same
through ipir_answer_batch with pinned host queries/responses (H2D + kernels +
D2H inside the timed region); plus the plain batch-1 q/s, p50/p99 latency of
the plain path, DB-pass GB/s, the roofline of the mat-vec kernel and the
CPU baseline (the oracle port on the host cores).

``--impl reference`` times the CPU restatement of the reference's server
path (the reference has no CPU server of its own) on a bounded sample of
the same workload.  Multi-GPU: every rank serves an independent replica.
"""
import argparse
import json
import os
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


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n-entries", type=int, default=1 << 29)
    ap.add_argument("--entry-bytes", type=int, default=30)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


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
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ CPU leg
def cpu_sample(params, seconds_hint=15.0):
    """Time the oracle port (CPU restatement of the server path) on a bounded
    sample of the workload and scale to q/s: mat-vec over a column slice,
    the tensor pass of a few groups, and the full Horner chain; the DB,
    precomp and query are synthetic (the work does not depend on values)."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import ctypes as C
    from oracle_lib import Oracle, ptr, u16p, u32p, u64p
    o = Oracle()
    threads = o.L.orc_num_threads()
    R, Ccols, G = params["db_rows"], params["db_cols"], params["n_packed"]
    D = min(params["interp_d"], G)
    rng = np.random.default_rng(5)
    # mat-vec on a slice of columns (all rows)
    cs = 2048
    db = rng.integers(0, 65535, R * cs, dtype=np.uint16)
    b = np.concatenate([rng.integers(0, Q[0], R, dtype=np.uint64), rng.integers(0, Q[1], R, dtype=np.uint64)])
    out = np.zeros(2 * cs, np.uint64)
    t0 = time.perf_counter()
    o.L.orc_matvec(ptr(db, u16p), R, cs, ptr(b, u64p), 0, cs, ptr(out, u64p))
    t_mv = (time.perf_counter() - t0) * (Ccols / cs)
    # tensor pass of sample groups (one at a time, as the CPU loop would)
    ng = 2
    dp = rng.integers(0, Q[0], 2 * NSTEPS * 2 * N, dtype=np.uint32)
    dm = rng.integers(0, Q[0], 2 * NSTEPS * 2 * N, dtype=np.uint32)
    df = rng.integers(0, Q[0], 2 * 2 * N, dtype=np.uint32)
    k5 = rng.integers(0, Q[0], 2 * 2 * N, dtype=np.uint64)
    kn = rng.integers(0, Q[0], 2 * 2 * N, dtype=np.uint64)
    r = rng.integers(0, Q[0], 2 * N, dtype=np.uint64)
    ob = np.zeros(2 * N, np.uint64)
    t0 = time.perf_counter()
    for _ in range(ng):
        o.L.orc_pack_group(ptr(r, u64p), N, 0, ptr(dp, u32p), ptr(dm, u32p), ptr(df, u32p),
                           ptr(k5, u64p), ptr(kn, u64p), ptr(ob, u64p))
    t_pack_1 = (time.perf_counter() - t0) / ng
    # groups run in parallel on the host threads
    t_pack = t_pack_1 * G / max(1, min(threads, G))
    # Horner chain of D cts (serial)
    L = min(D, 8)
    rg = np.concatenate([rng.integers(0, Q[(x // N) & 1], N, dtype=np.uint64) for x in range(0, 16 * N, N)])
    pk = np.concatenate([rng.integers(0, Q[(x // N) & 1], N, dtype=np.uint64) for x in range(0, 4 * N * L, N)])
    oh = np.zeros(4 * N, np.uint64)
    t0 = time.perf_counter()
    o.L.orc_horner(ptr(rg, u64p), ptr(pk, u64p), L, ptr(oh, u64p))
    t_h = (time.perf_counter() - t0) / max(1, L - 1) * max(0, D - 1) * params["num_cts"]
    per_query = t_mv + t_pack + t_h
    return {"value": 1.0 / per_query, "unit": "q/s", "cores": threads, "kind": "port",
            "sample": (f"oracle port on {threads} host threads: mat-vec over {cs} of {Ccols} columns x all "
                       f"{R} rows scaled by {Ccols // cs}; tensor pass of {ng} of {G} groups scaled to {G} "
                       f"groups over the threads; Horner {L - 1} of {D - 1} ExtProd steps scaled; "
                       f"per-query {per_query:.2f} s = mat-vec {t_mv:.2f} + tensor {t_pack:.2f} + Horner {t_h:.2f}")}


# ------------------------------------------------------------------ reference arm
def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    import inspire_b200 as ib
    params = ib.setup(args.n_entries, args.entry_bytes)
    vals = []
    for _ in range(max(1, args.warmup)):
        cpu_sample(params)
    for _ in range(args.steps):
        vals.append(cpu_sample(params)["value"])
    last = cpu_sample(params)
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": "q/s at 16 GB DB (CPU restatement of the reference server path)",
            "value": v, "unit": "q/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32/u64 modular",
            "data": "synthetic",
            "config": {"workload": "setup(2^29, w=30): 32768 x 262144 u16 DB (17.18 GB), 128 groups, batch 1",
                       "model": "InsPIRe PIR server", "global_batch": 1, "seq_len": 0, "parallelism": "replicas"},
            "cpu_baseline": {"value": v, "unit": "q/s", "cores": last["cores"], "kind": last["kind"],
                             "sample": last["sample"]},
            "e2e": {"value": v, "unit": "q/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
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
    params = ib.setup(args.n_entries, args.entry_bytes)
    R, Ccols, G, ncts = params["db_rows"], params["db_cols"], params["n_packed"], params["num_cts"]
    db = ib.fill_db(R * Ccols, 0)
    seed = bytes(range(64))
    t0 = time.perf_counter()
    srv = ib.Server(args.n_entries, args.entry_bytes, db, max_batch=max(B, 1), crs_seed=seed)
    t_pre = time.perf_counter() - t0
    del db
    # A dedicated stream: the handle of torch's default stream is 0, which the
    # C ABI reads as "the server's own stream".
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    srv.set_stream(stream.cuda_stream)
    qn = ib.query_u64s(params)
    rn = ib.response_u64s(params)
    qbuf_t = torch.empty((B, qn), dtype=torch.int64, pin_memory=True)
    qbuf = qbuf_t.numpy().view(np.uint64)
    synth_queries(params, B, 1000 + rank, qbuf)
    obuf_t = torch.empty((B, rn), dtype=torch.int64, pin_memory=True)
    obuf = obuf_t.numpy().view(np.uint64)
    views = (ib.IpirQueryView * B)()
    for i in range(B):
        views[i] = ib.query_view_from_flat(params, qbuf[i])

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    def device_time(count, steps):
        srv.stage_views(views, count)
        for _ in range(args.warmup):
            srv.run(count)
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            srv.run(count)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1) / steps)

    # stage timers (CUDA events on the launching stream) for the roofline
    srv.enable_stage_timing(True)
    srv.stage_views(views, 1)
    st1 = []
    for _ in range(max(3, args.warmup)):
        srv.run(1)
        srv.fetch(1, obuf[:1])
        st1.append(srv.stage_times())
    stB = []
    srv.stage_views(views, B)
    for _ in range(2):
        srv.run(B)
        srv.fetch(B, obuf)
        stB.append(srv.stage_times())
    srv.enable_stage_timing(False)

    # plain batch-1 device time
    ms1 = device_time(1, args.steps)
    # headline: served batch B, timed region sampled for clocks
    sampler = ClockSampler(local_rank)
    sampler.start()
    msB = device_time(B, args.steps)
    clocks = sampler.stop()
    value = world * B * 1000.0 / msB

    # e2e through the C ABI with pinned host buffers (H2D + kernels + D2H)
    for _ in range(args.warmup):
        srv.answer_batch_rc(views, B, obuf)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rc = srv.answer_batch_rc(views, B, obuf)
        assert rc == 0, ib.last_error()
    t_e2e = max_over_ranks((time.perf_counter() - t0) / args.steps)
    e2e_qps = world * B / t_e2e
    # plain path latency distribution (one query per call, e2e)
    lat = []
    for _ in range(max(args.steps, 20)):
        t0 = time.perf_counter()
        srv.answer_batch_rc(views, 1, obuf)
        lat.append((time.perf_counter() - t0) * 1000.0)
    lat.sort()
    p50 = lat[len(lat) // 2]
    p99 = lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))]

    mv1 = statistics.median(s["matvec"] for s in st1)
    db_bytes = R * Ccols * 2
    alg_bytes = db_bytes + 2 * R * 8          # DB + one query's b vector per launch
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (mv1 * 1e-3) / 1e9
    launches_per_step = 1 + (B + 3) // 4 + (B + 7) // 8 + 1 + 1
    tensor_bytes = G * 2 * (2 * NSTEPS * 2 * N * 4)

    line = {
        "metric": "q/s at 16 GB DB (served batch-32; plain batch-1, p50/p99 latency, DB-pass GB/s alongside)",
        "value": value, "unit": "q/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": msB, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32/u64 modular (exact)", "data": "synthetic",
        "config": {"workload": "setup(2^29, w=30): 32768 x 262144 u16 DB (17.18 GB), 128 groups, "
                               f"8.59 GB tensors, 1 ct/query; batch {B}",
                   "model": "InsPIRe PIR server", "global_batch": B * world, "seq_len": 0,
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (17 GB DB per step)"},
        "plain_b1": {"q_per_s": 1000.0 / ms1, "ms": ms1, "p50_ms_e2e": p50, "p99_ms_e2e": p99},
        "served": {"batch": B, "ms_per_batch": msB, "q_per_s": value / world},
        "db_pass_gbs": db_bytes / (mv1 * 1e-3) / 1e9,
        "stage_ms_b1": st1[-1], "stage_ms_batch": stB[-1],
        "preprocess_s": t_pre,
        "roofline": {"kernel": ("mv_tc_kernel (tcgen05 int8 DB pass, batch 1)" if os.environ.get("IPB_MATVEC", "tc") != "simt" else "matvec_kernel<1,8> (DB pass, batch 1)"), "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": None,
                     "alg_bytes_per_launch": alg_bytes},
        "tensor_pass_gbs_b1": tensor_bytes / (statistics.median(s["collapse"] for s in st1) * 1e-3) / 1e9,
        "e2e": {"value": e2e_qps, "unit": "q/s", "h2d_bytes_per_step": B * qn * 8,
                "d2h_bytes_per_step": B * rn * 8},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(params)
    srv.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
