"""Standalone exact mat-vec entry point (device pointers) against the
oracle's u128 CPU dot products on sampled columns, including a DB taller
than one 32768-row K-chunk and a multi-pass batch."""
import numpy as np
import pytest

from oracle_lib import Q0, Q1

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows,cols,count", [(2048, 4096, 1), (32768, 2048, 3), (65536, 1024, 33)])
def test_matvec_entry_point_matches_u128_oracle(rows, cols, count):
    import torch
    import inspire_b200 as ib
    g = torch.Generator(device="cuda").manual_seed(rows + cols + count)
    db = torch.randint(0, 65535, (rows * cols,), dtype=torch.int32, device="cuda", generator=g).to(torch.int16)
    q = torch.randint(-(2 ** 62), 2 ** 62, (count * 2 * rows,), dtype=torch.int64, device="cuda", generator=g)
    out = torch.zeros(count * 2 * cols, dtype=torch.int32, device="cuda")
    ib.matvec(db.data_ptr(), rows, cols, q.data_ptr(), count, out.data_ptr())
    torch.cuda.synchronize()
    dbh = db.cpu().numpy().view(np.uint16).reshape(rows, cols).astype(object)
    qh = q.cpu().numpy().view(np.uint64).reshape(count, 2, rows)
    oh = out.cpu().numpy().view(np.uint32).reshape(count, 2, cols)
    rng = np.random.default_rng(1)
    for qi in sorted({0, count - 1}):
        for l, mod in enumerate((Q0, Q1)):
            b = np.array([int(x) % mod for x in qh[qi, l]], dtype=object)
            for c in rng.integers(0, cols, 6):
                exp = int((dbh[:, c] * b).sum()) % mod
                assert int(oh[qi, l, c]) == exp, (qi, l, c)
