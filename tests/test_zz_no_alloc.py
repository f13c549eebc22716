"""The zero-allocation mat-vec entry point, for callers that may not
allocate device memory (their memory belongs to another allocator or pool,
or an allocation's implicit device synchronisation is not allowed there).
It must give exactly what the allocating entry point ipir_b200_matvec gives
(integer work: tolerance 0), on two calls in a row, since the second call
reuses the fixed scratch the first one left behind.  The first call runs on
a non-blocking stream, so the set-up copy of its tables must be ordered on
the caller's stream.  Sampled columns are also checked against exact u128
dot products.  This file is collected last so that a run stopping at the
first failure has run everything else."""
import numpy as np
import pytest

from oracle_lib import Q0, Q1

pytestmark = pytest.mark.gpu


def _inputs(rows, cols, count, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    db = torch.randint(0, 65535, (rows * cols,), dtype=torch.int32, device="cuda", generator=g).to(torch.int16)
    q = torch.randint(-(2 ** 62), 2 ** 62, (count * 2 * rows,), dtype=torch.int64, device="cuda", generator=g)
    return db, q


def _check_sampled_exact(db, q, out, rows, cols, count):
    dbh = db.cpu().numpy().view(np.uint16).reshape(rows, cols)
    qh = q.cpu().numpy().view(np.uint64).reshape(count, 2, rows)
    oh = out.cpu().numpy().view(np.uint32).reshape(count, 2, cols)
    cs = np.random.default_rng(rows + count).integers(0, cols, 12)
    d = dbh[:, cs].astype(np.uint64)                 # < 2^16
    for l, mod in enumerate((Q0, Q1)):
        b = qh[:, l, :] % np.uint64(mod)            # < 2^27: products < 2^43, sums < 2^59, exact in u64
        assert (oh[:, l, cs].astype(np.uint64) == (b @ d) % np.uint64(mod)).all(), l


@pytest.mark.parametrize("rows,cols,count", [(32768, 4096, 8), (2048, 2048, 1)])
def test_noalloc_matvec_equals_allocating_entry_point_twice(rows, cols, count):
    import torch
    import inspire_b200 as ib
    db, q = _inputs(rows, cols, count, rows + count)
    ref = torch.zeros(count * 2 * cols, dtype=torch.int32, device="cuda")
    ib.matvec(db.data_ptr(), rows, cols, q.data_ptr(), count, ref.data_ptr())
    torch.cuda.synchronize()
    side = torch.cuda.Stream()            # non-blocking with respect to the legacy default stream
    for call in range(2):
        out = torch.full((count * 2 * cols,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        stream = side.cuda_stream if call == 0 else 0
        rc = ib.matvec_noalloc_rc(db.data_ptr(), rows, cols, q.data_ptr(), count, out.data_ptr(), stream=stream)
        assert rc == 0, ib.last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, ref), f"call {call}: differs from ipir_b200_matvec"
    _check_sampled_exact(db, q, out, rows, cols, count)


def test_noalloc_rejects_shapes_beyond_its_scratch():
    import torch
    import inspire_b200 as ib
    db, q = _inputs(65536, 128, 1, 3)
    out = torch.zeros(2 * 128, dtype=torch.int32, device="cuda")
    assert ib.matvec_noalloc_rc(db.data_ptr(), 65536, 128, q.data_ptr(), 1, out.data_ptr()) == 2
    assert "32768" in ib.last_error()
    assert ib.matvec_noalloc_rc(db.data_ptr(), 2048, 128, q.data_ptr(), 9, out.data_ptr()) == 2
