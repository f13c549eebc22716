"""The zero-allocation mat-vec entry point, for callers that may not
allocate device memory (their memory belongs to another allocator or pool,
or an allocation's implicit device synchronisation is not allowed there).
It must give exactly what the allocating entry point ipir_b200_matvec gives
(integer work: tolerance 0), on two calls in a row, since the second call
reuses the fixed scratch the first one left behind.  This file is collected
last so that a run stopping at the first failure has run everything else."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _inputs(rows, cols, count, seed):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    db = torch.randint(0, 65535, (rows * cols,), dtype=torch.int32, device="cuda", generator=g).to(torch.int16)
    q = torch.randint(-(2 ** 62), 2 ** 62, (count * 2 * rows,), dtype=torch.int64, device="cuda", generator=g)
    return db, q


@pytest.mark.parametrize("rows,cols,count", [(32768, 4096, 8), (2048, 2048, 1)])
def test_noalloc_matvec_equals_allocating_entry_point_twice(rows, cols, count):
    import torch
    import inspire_b200 as ib
    db, q = _inputs(rows, cols, count, rows + count)
    ref = torch.zeros(count * 2 * cols, dtype=torch.int32, device="cuda")
    ib.matvec(db.data_ptr(), rows, cols, q.data_ptr(), count, ref.data_ptr())
    for call in range(2):
        out = torch.full((count * 2 * cols,), -1, dtype=torch.int32, device="cuda")
        rc = ib.matvec_noalloc_rc(db.data_ptr(), rows, cols, q.data_ptr(), count, out.data_ptr())
        assert rc == 0, ib.last_error()
        torch.cuda.synchronize()
        assert torch.equal(out, ref), f"call {call}: differs from ipir_b200_matvec"


def test_noalloc_rejects_shapes_beyond_its_scratch():
    import torch
    import inspire_b200 as ib
    db, q = _inputs(65536, 128, 1, 3)
    out = torch.zeros(2 * 128, dtype=torch.int32, device="cuda")
    assert ib.matvec_noalloc_rc(db.data_ptr(), 65536, 128, q.data_ptr(), 1, out.data_ptr()) == 2
    assert "32768" in ib.last_error()
    assert ib.matvec_noalloc_rc(db.data_ptr(), 2048, 128, q.data_ptr(), 9, out.data_ptr()) == 2
