"""The tensor-core kernels' abort path, exercised without a fault.  A test
hook (IPB_TEST_ABORT_AFTER_ITEMS, read at each launch) makes the MMA
issuer of mv_tc_kernel and tp_tc_kernel stop after a few work items, the
path a bounded wait that runs out takes.  The other roles leave at once
(their waits watch the CTA's abort flag), the producer still waits for the
loads it issued and the MMA issuer for the MMAs it issued before TMEM is
released.  Each call must return its error code promptly, write nothing
into the caller's buffer, and leave the context usable: the next call
without the hook gives the exact answer."""
import os
import time

import numpy as np
import pytest

from cases import get_case
from oracle_lib import Q0, Q1

pytestmark = pytest.mark.gpu


@pytest.fixture
def abort_hook():
    os.environ["IPB_TEST_ABORT_AFTER_ITEMS"] = "2"
    yield
    os.environ.pop("IPB_TEST_ABORT_AFTER_ITEMS", None)


def test_matvec_abort_reports_and_recovers(abort_hook):
    import torch
    import inspire_b200 as ib
    rows, cols, count = 32768, 16384, 8
    g = torch.Generator(device="cuda").manual_seed(3)
    db = torch.randint(0, 65535, (rows * cols,), dtype=torch.int32, device="cuda", generator=g).to(torch.int16)
    q = torch.randint(0, 2 ** 40, (count * 2 * rows,), dtype=torch.int64, device="cuda", generator=g)
    out = torch.zeros(count * 2 * cols, dtype=torch.int32, device="cuda")
    t0 = time.perf_counter()
    with pytest.raises(ib.InspireError) as e:
        ib.matvec_ex(db.data_ptr(), rows, cols, q.data_ptr(), count, out.data_ptr(), path=0)
    assert "rc=5" in str(e.value) and "code 99" in str(e.value)
    assert time.perf_counter() - t0 < 20.0                 # the other roles left without running out their limits
    os.environ.pop("IPB_TEST_ABORT_AFTER_ITEMS")
    ib.matvec_ex(db.data_ptr(), rows, cols, q.data_ptr(), count, out.data_ptr(), path=0)
    torch.cuda.synchronize()
    dbh = db.cpu().numpy().view(np.uint16).reshape(rows, cols)
    qh = q.cpu().numpy().view(np.uint64).reshape(count, 2, rows)
    oh = out.cpu().numpy().view(np.uint32).reshape(count, 2, cols)
    cs = np.random.default_rng(4).integers(0, cols, 16)
    d = dbh[:, cs].astype(np.uint64)
    for l, mod in enumerate((Q0, Q1)):
        b = qh[:, l, :] % np.uint64(mod)
        assert (oh[:, l, cs].astype(np.uint64) == (b @ d) % np.uint64(mod)).all(), l


def test_answer_abort_writes_nothing_and_recovers(abort_hook):
    import inspire_b200 as ib
    c = get_case("batch")
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=4, crs_seed=c.seed)
    try:
        qs = [c.query(i, 8100 + k)[0] for k, i in enumerate([5, 77777, 524287])]
        views = (ib.IpirQueryView * 3)()
        keep = [np.ascontiguousarray(x) for x in qs]
        for i, f in enumerate(keep):
            views[i] = ib.query_view_from_flat(srv.params, f)
        out = np.full((3, ib.response_u64s(srv.params)), 7, np.uint64)
        t0 = time.perf_counter()
        assert srv.answer_batch_rc(views, 3, out) == 4
        assert "code 99" in ib.last_error()
        assert time.perf_counter() - t0 < 20.0
        assert (out == 7).all()                             # nothing written
        os.environ.pop("IPB_TEST_ABORT_AFTER_ITEMS")
        assert srv.answer_batch_rc(views, 3, out) == 0
        for k in range(3):
            assert (out[k] == c.oracle_answer(qs[k])).all(), k
    finally:
        srv.close()


@pytest.mark.parametrize("hc", [1, 2])
def test_chunked_pipeline_abort_writes_nothing_and_recovers(abort_hook, hc):
    """The same with the Horner chain trailing the DB pass in chunks (128
    groups, 8 chunks): the mat-vec and tensor-pass launches stop early while
    the Horner stream keeps consuming chunks; the blocking answer and the
    staged path both report the error with nothing written, and the next
    calls without the hook give the unchunked answers."""
    import inspire_b200 as ib
    c = get_case("g128")
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=2, crs_seed=c.seed)
    try:
        os.environ.pop("IPB_TEST_ABORT_AFTER_ITEMS")
        qs = [c.query(i, 8200 + k)[0] for k, i in enumerate([9, 8000000])]
        for n in (1, 2):
            srv.set_schedule(n, matvec_tc=1, horner_cluster=hc)
        want = srv.answer_batch(qs)
        for n in (1, 2):
            srv.set_schedule(n, matvec_tc=1, horner_cluster=hc, hchunks=8)
        views = (ib.IpirQueryView * 2)()
        keep = [np.ascontiguousarray(x) for x in qs]
        for i, f in enumerate(keep):
            views[i] = ib.query_view_from_flat(srv.params, f)
        out = np.full((2, ib.response_u64s(srv.params)), 7, np.uint64)
        os.environ["IPB_TEST_ABORT_AFTER_ITEMS"] = "2"
        t0 = time.perf_counter()
        assert srv.answer_batch_rc(views, 2, out) == 4
        assert "code 99" in ib.last_error()
        assert (out == 7).all()
        srv.stage_views(views, 1)
        srv.run(1)
        with pytest.raises(ib.InspireError):
            srv.fetch(1, out[:1])
        assert (out == 7).all()
        assert time.perf_counter() - t0 < 40.0
        os.environ.pop("IPB_TEST_ABORT_AFTER_ITEMS")
        assert srv.answer_batch_rc(views, 2, out) == 0
        assert (out == want).all()
        assert (srv.answer(qs[1]) == want[1]).all()
    finally:
        srv.close()
