"""The Horner chain trailing the DB pass in group chunks (schedule field
hchunks: at most that many chunks): the tensor pass first, then the mat-vec
and finalize chunk by chunk from the top group down, each chunk's Horner
steps on a second stream resuming the chain from memory.  The chunks are
whole waves of mat-vec work growing by one wave per chunk from the bottom
(at 128 groups on 148 SMs: 119 + 9, 101 + 18 + 9 and 37 + 37 + 27 + 18 + 9
for at most 2, 3 and 8 chunks; 4 + 4 at 8 groups).  Every chunking, with both cluster Horner kernels, through the blocking
answer (host views), the staged path (stage_views / run / fetch) and stage
timing (which runs unchunked), gives the unchunked responses bit for bit,
and those are pinned to the oracle and to extract()."""
import numpy as np
import pytest

from cases import get_case

pytestmark = pytest.mark.gpu


def _staged(ib, srv, qs):
    n = len(qs)
    flat = np.ascontiguousarray(np.stack(qs))
    views = (ib.IpirQueryView * n)()
    for i in range(n):
        views[i] = ib.query_view_from_flat(srv.params, flat[i])
    srv.stage_views(views, n)
    srv.run(n)
    out = np.zeros((n, ib.response_u64s(srv.params)), np.uint64)
    srv.fetch(n, out)
    return out


@pytest.mark.parametrize("name,idx,chunks", [
    ("batch", [0, 42, 1000, 100000, 524287, 0, 42, 1000], (2, 8)),          # G = 8
    ("g128", [0, 5, 777777, 8388607], (2, 3, 8)),                           # G = 128: the 16 GB group count
])
def test_chunked_horner_equals_unchunked(name, idx, chunks):
    import inspire_b200 as ib
    c = get_case(name)
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=len(idx), crs_seed=c.seed)
    try:
        assert srv.params["num_cts"] == 1
        qs, sts = [], []
        for k, i in enumerate(idx):
            q, st = c.query(i, 7100 + k)
            qs.append(q)
            sts.append(st)
        sizes = sorted({1, 2, len(idx)})
        for n in sizes:
            srv.set_schedule(n, matvec_tc=1, horner_cluster=1)
        want = {n: srv.answer_batch(qs[:n]) for n in sizes}
        for n in sizes:
            assert (want[n] == want[len(idx)][:n]).all()
        assert (want[1][0] == c.oracle_answer(qs[0])).all()
        for i, st in enumerate(sts):
            assert (st.extract(want[len(idx)][i]) == c.expected_slots(idx[i])).all(), i
        for hc in (1, 2):
            for k in chunks:
                for n in sizes:
                    srv.set_schedule(n, matvec_tc=1, horner_cluster=hc, hchunks=k)
                    assert srv.schedule(n)["hchunks"] == k
                    assert (srv.answer_batch(qs[:n]) == want[n]).all(), (hc, k, n, "blocking")
                    assert (_staged(ib, srv, qs[:n]) == want[n]).all(), (hc, k, n, "staged")
                    assert (srv.answer_batch(qs[:n]) == want[n]).all(), (hc, k, n, "again")
            srv.enable_stage_timing(True)
            assert (srv.answer_batch(qs) == want[len(idx)]).all(), (hc, "timed")
            srv.enable_stage_timing(False)
        with pytest.raises(Exception):
            srv.set_schedule(1, matvec_tc=1, horner_cluster=1, hchunks=17)
    finally:
        srv.close()


def test_chunked_full_pass_of_32_queries():
    """32 queries at 128 groups (one whole mat-vec pass, 32 chains of 4- or
    8-CTA clusters trailing it, 29 leaving a ragged last block): chunked
    equals unchunked for both cluster kernels."""
    import inspire_b200 as ib
    c = get_case("g128")
    idx = [int(i) for i in np.random.default_rng(21).integers(0, c.n_entries, 32)]
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=32, crs_seed=c.seed)
    try:
        qs = [c.query(i, 7400 + k)[0] for k, i in enumerate(idx)]
        for n in (29, 32):
            srv.set_schedule(n, matvec_tc=1, horner_cluster=1)
        want = srv.answer_batch(qs)
        assert (srv.answer_batch(qs[:29]) == want[:29]).all()
        for hc in (1, 2):
            for n in (29, 32):
                srv.set_schedule(n, matvec_tc=1, horner_cluster=hc, hchunks=8)
            assert (srv.answer_batch(qs) == want).all(), hc
            assert (_staged(ib, srv, qs[:29]) == want[:29]).all(), hc
    finally:
        srv.close()


def test_chunking_ignored_where_it_does_not_apply():
    """The one-CTA Horner kernel, the tensor pass beside the mat-vec and the
    CUDA-core mat-vec do not chunk: with hchunks set they run the plain
    pipeline and still give the same responses."""
    import inspire_b200 as ib
    c = get_case("batch")
    idx = [3, 99, 4096]
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=3, crs_seed=c.seed)
    try:
        qs = [c.query(i, 7200 + k)[0] for k, i in enumerate(idx)]
        want = srv.answer_batch(qs)
        for kw in (dict(matvec_tc=1, horner_cluster=0), dict(matvec_tc=1, horner_cluster=1, tp_sms=40),
                   dict(matvec_tc=0, horner_cluster=2)):
            srv.set_schedule(3, hchunks=4, **kw)
            assert (srv.answer_batch(qs) == want).all(), kw
    finally:
        srv.close()
