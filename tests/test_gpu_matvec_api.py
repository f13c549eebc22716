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


@pytest.mark.parametrize("path,qpp,kchunk", [(0, 0, 0), (0, 8, 8192), (0, 3, 32768), (1, 0, 0), (1, 3, 0)])
def test_matvec_schedules_match_u128_oracle(path, qpp, kchunk):
    """Every schedule of ipir_b200_matvec_ex (tensor cores with several pass
    sizes and K-chunks, CUDA cores) gives the exact sums."""
    import torch
    import inspire_b200 as ib
    rows, cols, count = 65536, 4096, 9
    g = torch.Generator(device="cuda").manual_seed(77 + path + qpp)
    db = torch.empty(rows * cols, dtype=torch.int16, device="cuda")
    ib.fill_db_device(db.data_ptr(), rows * cols, 12345)
    q = torch.randint(-(2 ** 62), 2 ** 62, (count * 2 * rows,), dtype=torch.int64, device="cuda", generator=g)
    out = torch.zeros(count * 2 * cols, dtype=torch.int32, device="cuda")
    ib.matvec_ex(db.data_ptr(), rows, cols, q.data_ptr(), count, out.data_ptr(), path=path, queries_per_pass=qpp,
                 kchunk_rows=kchunk)
    torch.cuda.synchronize()
    dbh = db.cpu().numpy().view(np.uint16).reshape(rows, cols)
    qh = q.cpu().numpy().view(np.uint64).reshape(count, 2, rows)
    oh = out.cpu().numpy().view(np.uint32).reshape(count, 2, cols)
    cs = np.random.default_rng(path).integers(0, cols, 16)
    d = dbh[:, cs].astype(np.uint64)                     # < 2^16
    for l, mod in enumerate((Q0, Q1)):
        b = qh[:, l, :] % np.uint64(mod)                # < 2^27: products < 2^43, sums < 2^59
        exp = (b @ d) % np.uint64(mod)                  # exact in u64
        assert (oh[:, l, cs].astype(np.uint64) == exp).all(), l


def test_fill_db_device_matches_host():
    import torch
    import inspire_b200 as ib
    n = 1_000_003
    d = torch.empty(n, dtype=torch.int16, device="cuda")
    ib.fill_db_device(d.data_ptr(), n, 99)
    torch.cuda.synchronize()
    assert (d.cpu().numpy().view(np.uint16) == ib.fill_db(n, 99)).all()
