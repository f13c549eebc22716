"""Group sharding on the GPU (ipir_b200_shard_* / ipir_b200_horner_*): a
database split into 2 and 3 group shards (uneven ranges included) on one
device, their packed b parts placed in group order as the NCCL gather
places them, and the Horner owner's responses must equal
ipir_answer_batch's on the whole database (integer work: tolerance 0), for
geometries with one and two response ciphertexts' worth of groups and a
batch over 32 queries; plus the torch.distributed form (ShardedServer) on a
one-rank NCCL group."""
import numpy as np
import pytest

from cases import get_case

pytestmark = pytest.mark.gpu


def _sharded_answer(ib, c, nshards, qs):
    import torch
    ranges = ib.group_ranges(c.G, nshards)
    shards = [ib.Shard(c.n_entries, c.w, c.db, lo, hi, c.seed, db_rows=c.db_rows_arg, max_batch=len(qs))
              for lo, hi in ranges]
    try:
        a_all = np.concatenate([s.export_a() for s in shards])
        packed = torch.empty((len(qs), c.G, 2 * 2048), dtype=torch.int32, device="cuda")
        for s, (lo, hi) in zip(shards, ranges):
            part = torch.empty((len(qs), hi - lo, 2 * 2048), dtype=torch.int32, device="cuda")
            s.pack(qs, part.data_ptr())
            packed[:, lo:hi] = part
        owner = ib.HornerOwner(shards[0].params, a_all, max_batch=len(qs))
        try:
            return owner.answer(packed.data_ptr(), qs, stream=torch.cuda.current_stream().cuda_stream)
        finally:
            owner.close()
    finally:
        for s in shards:
            s.close()


@pytest.mark.parametrize("name,nshards,nq", [("batch", 2, 3), ("batch", 3, 3), ("medium", 3, 2), ("g128", 2, 34)])
def test_shards_equal_the_whole_server(name, nshards, nq):
    import inspire_b200 as ib
    c = get_case(name)
    idx = [(7919 * k + 13) % c.n_entries for k in range(nq)]
    qs = [c.query(i, 900 + k)[0] for k, i in enumerate(idx)]
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=c.db_rows_arg, max_batch=nq, crs_seed=c.seed)
    try:
        want = srv.answer_batch(qs)
    finally:
        srv.close()
    got = _sharded_answer(ib, c, nshards, qs)
    assert (got == want).all()


def test_sharded_server_on_a_one_rank_nccl_group():
    import datetime
    import os
    import socket
    import torch
    import torch.distributed as dist
    import inspire_b200 as ib
    from inspire_b200.sharded import ShardedServer
    c = get_case("batch")
    qs = [c.query(i, 950 + k)[0] for k, i in enumerate([3, 524287])]
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=2, crs_seed=c.seed)
    want = srv.answer_batch(qs)
    srv.close()
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        ss = ShardedServer(c.n_entries, c.w, c.db, c.seed, db_rows=2048, max_batch=2)
        got = ss.answer_batch(qs)
        ss.close()
        assert (got == want).all()
    finally:
        dist.destroy_process_group()


def test_whole_chunk_shards_answer_their_own_ciphertexts():
    """A database of two response ciphertexts (G = 512 groups, D = 256) in
    two shards of whole Horner chunks: each answers its own ciphertext with
    no exchange, and the two side by side are the whole server's response;
    a shard that does not cover whole chunks refuses (code 6)."""
    import inspire_b200 as ib
    c = get_case("g512")
    qs = [c.query(i, 990 + k)[0] for k, i in enumerate([11, 33554431])]
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=2, crs_seed=c.seed)
    try:
        want = srv.answer_batch(qs)
    finally:
        srv.close()
    ranges = ib.chunk_ranges(c.G, min(c.D, c.G), 2)
    assert ranges == [(0, 256), (256, 512)]
    parts = []
    for lo, hi in ranges:
        sh = ib.Shard(c.n_entries, c.w, c.db, lo, hi, c.seed, db_rows=2048, max_batch=2)
        try:
            assert sh.cts() == 1
            parts.append(sh.answer(qs))
        finally:
            sh.close()
    assert (np.concatenate(parts, axis=1) == want).all()
    sh = ib.Shard(c.n_entries, c.w, c.db, 0, 100, c.seed, db_rows=2048, max_batch=2)
    try:
        assert sh.cts() == 0
        with pytest.raises(ib.InspireError, match="rc=6"):
            sh.answer(qs)
    finally:
        sh.close()
