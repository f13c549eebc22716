"""Group sharding's host logic on CPU: two (and three) gloo ranks on
127.0.0.1.  Each rank computes, with the oracle, only its groups' part of
the answer -- the mat-vec over its column range and the per-group pack of
its groups (src/gpu_protocol.cu:1225-1283) -- and the package's own gather
functions (inspire_b200.sharded.gather_a / gather_packed, the ones the GPU
path runs over NCCL) bring the parts to the owner, which runs the Horner
chains (src/crypto.cpp:264-279) and must reproduce the single-process
oracle answer bit for bit, for several queries, uneven ranges included."""
import os
import socket
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import datetime, os, sys
sys.path.insert(0, os.path.join({repo!r}, "inspire-gpu_b200"))
sys.path.insert(0, os.path.join({repo!r}, "tests"))
import numpy as np, torch, torch.distributed as dist
from inspire_b200 import group_ranges
from inspire_b200.sharded import gather_a, gather_packed
from cases import get_case
from oracle_lib import N, PRE_A, PRE_D, PRE_F, QS, ptr, u32p, u64p

rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
c = get_case({case!r})
o, R, C, G, D = c.o, c.R, c.C, c.G, c.D
ranges = group_ranges(G, world)
lo, hi = ranges[rank]
gmax = max(h - l for l, h in ranges)
dbe, (pa, pdp, pdm, pdf) = c.pre           # this test's ranks share the oracle precomp
qs = [c.query(i, 500 + k)[0] for k, i in enumerate({idx!r})]

def keys_ntt(q):
    blk = 2 * 2 * N
    k5 = np.zeros(2 * 2 * N, np.uint64)
    kn = np.zeros(2 * 2 * N, np.uint64)
    for j in range(2):
        for l in range(2):
            src = slice(2 * R + (j * 2 + l) * N, 2 * R + (j * 2 + l + 1) * N)
            dst = slice((l * 2 + j) * N, (l * 2 + j + 1) * N)
            k5[dst] = o.ntt_forward(q[src] % np.uint64(QS[l]), l)
            k5n = q[2 * R + blk:][(j * 2 + l) * N:(j * 2 + l + 1) * N]
            kn[dst] = o.ntt_forward(k5n % np.uint64(QS[l]), l)
    return k5, kn

local = torch.zeros((len(qs), gmax, 2 * N), dtype=torch.int32)
for k, q in enumerate(qs):
    b = np.concatenate([q[:R] % np.uint64(QS[0]), q[R:2 * R] % np.uint64(QS[1])])
    r = o.matvec(dbe, R, C, b, col_lo=lo * N, col_hi=hi * N)   # this rank's columns only
    k5, kn = keys_ntt(q)
    for g in range(lo, hi):
        out = np.zeros(2 * N, np.uint64)
        o.L.orc_pack_group(ptr(r, u64p), C, g, ptr(pdp[g * PRE_D:(g + 1) * PRE_D], u32p),
                           ptr(pdm[g * PRE_D:(g + 1) * PRE_D], u32p), ptr(pdf[g * PRE_F:(g + 1) * PRE_F], u32p),
                           ptr(k5, u64p), ptr(kn, u64p), ptr(out, u64p))
        local[k, g - lo] = torch.from_numpy(out.astype(np.uint32).view(np.int32))
a_all = gather_a(pa[lo * PRE_A:hi * PRE_A].copy(), ranges, rank, 0, dist)
packed = gather_packed(local, ranges, rank, 0, len(qs), dist)
if rank == 0:
    assert (a_all == pa).all()
    Da = min(D, G)
    for k, q in enumerate(qs):
        x = np.arange(4 * 2 * 2 * N)
        rgsw = q[2 * R + 2 * 2 * 2 * N:] % np.where(((x // N) & 1) == 1, QS[1], QS[0]).astype(np.uint64)
        cts = np.zeros((G, 4 * N), np.uint64)            # [group][a | b][limb][N]
        cts[:, :2 * N] = a_all.reshape(G, 2 * N)
        cts[:, 2 * N:] = packed[k].numpy().view(np.uint32).reshape(G, 2 * N)
        got = np.concatenate([o.horner(rgsw, np.ascontiguousarray(cts[s:s + Da]).reshape(-1), Da)
                              for s in range(0, G, Da)])
        want = c.oracle_answer(q)
        assert (got == want).all(), k
    print("RANK0 ok", flush=True)
dist.barrier()
dist.destroy_process_group()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("case,world,idx", [("batch", 2, [1, 300000, 524287]), ("medium", 3, [42, 42]),
                                            ("medium", 2, [7, 262143])])
def test_sharded_gather_reproduces_the_single_process_answer(tmp_path, case, world, idx):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(repo=REPO, case=case, idx=idx))
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="2")
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        out, _ = p.communicate(timeout=300)
        outs.append(out)
    for p, out in zip(procs, outs):
        assert p.returncode == 0, out[-3000:]
    assert "RANK0 ok" in outs[0]


CHUNK_WORKER = r"""
import datetime, os, sys
sys.path.insert(0, os.path.join({repo!r}, "inspire-gpu_b200"))
import numpy as np, torch.distributed as dist
from inspire_b200 import chunk_ranges
from inspire_b200.sharded import gather_responses
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
ranges = chunk_ranges(1300, 256, world)          # 6 ciphertexts, the last of 20 groups
cts = [-(-(h - l) // 256) for l, h in ranges]
full = np.random.default_rng(1).integers(0, 2 ** 27, (3, 6 * 4 * 2048), dtype=np.uint64)
lo_ct = ranges[rank][0] // 256
own = full[:, lo_ct * 4 * 2048:(lo_ct + cts[rank]) * 4 * 2048]
got = gather_responses(own, cts, rank, 0, dist)
if rank == 0:
    assert sum(cts) == 6 and ranges[-1][1] == 1300
    assert (got == full).all()
    print("RANK0 ok", flush=True)
dist.barrier()
dist.destroy_process_group()
"""


@pytest.mark.parametrize("world", [2, 4])
def test_chunk_shards_gather_responses_in_ciphertext_order(tmp_path, world):
    script = tmp_path / "chunk_worker.py"
    script.write_text(CHUNK_WORKER.format(repo=REPO))
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=120)[0] for p in procs]
    for p, out in zip(procs, outs):
        assert p.returncode == 0, out[-3000:]
    assert "RANK0 ok" in outs[0]
