"""One database over several GPUs, split by contiguous group ranges: one
process per GPU in a torch.distributed process group (NCCL over NVLink),
each holding a Shard; the owner rank also holds the HornerOwner.

Per batch (every rank calls answer_batch with the same queries):
  1. each rank's shard computes the b parts of its groups' packed
     ciphertexts (mat-vec over its column slab, tensor pass, finalize);
  2. one gather of those parts to the owner (2 N u32 per group and query;
     ranks with fewer groups pad to the largest range);
  3. the owner places them in group order and runs the Horner chains.
For databases of several response ciphertexts (64 GB and up) the ranks can
instead hold whole Horner chunks (mode "chunks"): each answers its own
ciphertexts and only finished responses are gathered.  Either way the
responses equal the single-GPU server's.  There is no counterpart in the
reference, which runs on one GPU (docs/ARCHITECTURE.md:32).
"""
import numpy as np

from . import RING_N, HornerOwner, Shard, chunk_ranges, group_ranges, setup


def gather_packed(local, ranges, rank, owner, count, dist, group=None):
    """Gather every rank's packed b parts to `owner`.

    local: tensor [>= count, gmax, 2 N] (int32) holding this rank's groups
    first (gmax = the largest range).  Returns, on the owner, a contiguous
    tensor [count, n_groups, 2 N] in global group order; None elsewhere.
    Every rank takes part in the one collective (same shapes everywhere)."""
    import torch
    gmax = max(hi - lo for lo, hi in ranges)
    send = local[:count].contiguous()
    assert send.shape[1] == gmax, (send.shape, gmax)
    bufs = [torch.empty_like(send) for _ in ranges] if rank == owner else None
    dist.gather(send, gather_list=bufs, dst=owner, group=group)
    if rank != owner:
        return None
    n_groups = ranges[-1][1]
    out = torch.empty((count, n_groups, send.shape[2]), dtype=send.dtype, device=send.device)
    for (lo, hi), b in zip(ranges, bufs):
        out[:, lo:hi] = b[:, : hi - lo]
    return out


def gather_a(a_local, ranges, rank, owner, dist, group=None):
    """Gather the shards' a parts ([groups][2 N] u32 each) to the owner, once
    at set-up; returns the host array [n_groups * 2 N] u32 on the owner."""
    import torch
    gmax = max(hi - lo for lo, hi in ranges)
    lo, hi = ranges[rank]
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    send = torch.zeros((gmax, 2 * RING_N), dtype=torch.int32, device=dev)
    send[: hi - lo] = torch.from_numpy(a_local.view(np.int32).reshape(hi - lo, 2 * RING_N)).to(dev)
    bufs = [torch.empty_like(send) for _ in ranges] if rank == owner else None
    dist.gather(send, gather_list=bufs, dst=owner, group=group)
    if rank != owner:
        return None
    parts = [b[: h - l].cpu().numpy().view(np.uint32) for (l, h), b in zip(ranges, bufs)]
    return np.ascontiguousarray(np.concatenate(parts).reshape(-1))


def gather_responses(resp, cts, rank, owner, dist, group=None):
    """Gather the ranks' own ciphertexts of each query's response (whole-chunk
    shards) to `owner`, in rank order = ciphertext order; returns the host
    array (count, n_cts * 4 N) u64 on the owner, None elsewhere."""
    import torch
    count = resp.shape[0]
    cmax = max(cts)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    send = torch.zeros((count, cmax * 4 * RING_N), dtype=torch.int64, device=dev)
    send[:, : resp.shape[1]] = torch.from_numpy(np.ascontiguousarray(resp).view(np.int64)).to(dev)
    bufs = [torch.empty_like(send) for _ in cts] if rank == owner else None
    dist.gather(send, gather_list=bufs, dst=owner, group=group)
    if rank != owner:
        return None
    parts = [b[:, : c * 4 * RING_N].cpu().numpy().view(np.uint64) for c, b in zip(cts, bufs)]
    return np.ascontiguousarray(np.concatenate(parts, axis=1))


class ShardedServer:
    """A database split over the ranks of `group` (default: the world), one
    rank per GPU, each on its current CUDA device; rank `owner` answers.

    db: the whole host DB (every rank preprocesses only its column slab);
    crs_seed: the 64-byte CRS seed, the same on every rank.
    mode "groups": contiguous group ranges, one gather of packed ciphertexts
    before the owner's Horner chains; mode "chunks" (databases of at least
    as many response ciphertexts as ranks): each rank holds whole Horner
    chunks and answers its own ciphertexts, and only the finished responses
    are gathered."""

    def __init__(self, n_entries, entry_bytes, db, crs_seed, db_rows=0, max_batch=16, owner=0, group=None,
                 mode="groups"):
        import torch
        import torch.distributed as dist
        self.dist, self.group, self.owner, self.mode = dist, group, owner, mode
        self.rank, world = dist.get_rank(group), dist.get_world_size(group)
        params = setup(n_entries, entry_bytes, db_rows)
        if mode == "chunks":
            self.ranges = chunk_ranges(params["n_packed"], min(params["interp_d"], params["n_packed"]), world)
        elif mode == "groups":
            self.ranges = group_ranges(params["n_packed"], world)
        else:
            raise ValueError("mode must be 'groups' or 'chunks'")
        lo, hi = self.ranges[self.rank]
        self.shard = Shard(n_entries, entry_bytes, db, lo, hi, crs_seed, db_rows=db_rows, max_batch=max_batch)
        self.params = self.shard.params
        self.max_batch = max_batch
        if mode == "chunks":
            d_act = min(params["interp_d"], params["n_packed"])
            self.cts = [-(-(h - l) // d_act) for l, h in self.ranges]
            self.horner = None
            return
        gmax = max(h - l for l, h in self.ranges)
        self.local = torch.zeros((max_batch, gmax, 2 * RING_N), dtype=torch.int32, device="cuda")
        # a shard with fewer groups than the largest packs densely here, then
        # pads into `local` (the gather needs equal shapes)
        self.dense = None if hi - lo == gmax else torch.empty((max_batch, hi - lo, 2 * RING_N), dtype=torch.int32,
                                                              device="cuda")
        a_all = gather_a(self.shard.export_a(), self.ranges, self.rank, owner, dist, group)
        self.horner = HornerOwner(self.params, a_all, max_batch) if self.rank == owner else None

    def answer_batch(self, queries):
        """Every rank passes the same flat queries; returns the responses
        (count, num_cts * 4 N) u64 on the owner, None on the other ranks."""
        import torch
        count = len(queries)
        if count > self.max_batch:
            raise ValueError("count exceeds max_batch")
        if self.mode == "chunks":
            own = self.shard.answer(queries)
            return gather_responses(own, self.cts, self.rank, self.owner, self.dist, self.group)
        if self.dense is None:
            self.shard.pack(queries, self.local.data_ptr())
        else:
            self.shard.pack(queries, self.dense.data_ptr())
            self.local[:count, : self.dense.shape[1]] = self.dense[:count]
        packed = gather_packed(self.local, self.ranges, self.rank, self.owner, count, self.dist, self.group)
        if self.rank != self.owner:
            return None
        return self.horner.answer(packed.data_ptr(), queries, stream=torch.cuda.current_stream().cuda_stream)

    def close(self):
        self.shard.close()
        if self.horner is not None:
            self.horner.close()
