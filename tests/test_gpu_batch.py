"""gpu_answer_batch contract (reference tests/test_gpu_batch.cu): batch ==
independent single answers bit-exact, slot-exact extract, caps consistent,
rerun reproducible, partial batches, duplicate indices with fresh keys;
plus the C-ABI error codes with nothing written (tests/test_capi.cu:110-114)."""
import ctypes as C

import numpy as np
import pytest

from cases import get_case

pytestmark = pytest.mark.gpu

IDX = [0, 42, 1000, 100000, 524287, 0, 42, 1000, 100000, 524287]


@pytest.fixture(scope="module")
def batch_env():
    import inspire_b200 as ib
    c = get_case("batch")
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=10, crs_seed=c.seed)
    qs, sts = [], []
    for k, idx in enumerate(IDX):
        q, st = c.query(idx, 3000 + k)   # fresh key material per query
        qs.append(q)
        sts.append(st)
    yield c, srv, qs, sts
    srv.close()


def test_caps(batch_env):
    c, srv, _, _ = batch_env
    caps = srv.caps()
    assert caps["max_batch"] == 10 and caps["num_cts"] == c.ncts and caps["resident_bytes"] > 0
    assert caps["device_free_bytes"] > 0


def test_batch_equals_singles_and_oracle(batch_env):
    c, srv, qs, sts = batch_env
    singles = np.stack([srv.answer(q) for q in qs])
    batch = srv.answer_batch(qs)
    assert (batch == singles).all()
    for i in (0, 4, 9):
        assert (batch[i] == c.oracle_answer(qs[i])).all(), i
    for i, st in enumerate(sts):
        assert (st.extract(batch[i]) == c.expected_slots(IDX[i])).all(), i
    # duplicate indices, fresh keys: different ciphertexts, same plaintext
    assert not (batch[0] == batch[5]).all()
    again = srv.answer_batch(qs)
    assert (again == batch).all()
    for n in (3, 2):
        part = srv.answer_batch(qs[:n])
        assert (part == singles[:n]).all()


def test_capi_error_codes_write_nothing(batch_env):
    import inspire_b200 as ib
    c, srv, qs, _ = batch_env
    views = (ib.IpirQueryView * 11)()
    keep = [np.ascontiguousarray(q) for q in qs] + [np.ascontiguousarray(qs[0])]
    for i, f in enumerate(keep):
        views[i] = ib.query_view_from_flat(srv.params, f)
    out = np.full((11, ib.response_u64s(srv.params)), 7, np.uint64)
    assert srv.answer_batch_rc(views, 11, out) == 2          # count > max_batch
    assert (out == 7).all()
    bad = (ib.IpirQueryView * 2)()
    bad[0] = views[0]
    bad[1] = views[1]
    bad[1].rgsw = C.cast(0, ib.u64p)
    assert srv.answer_batch_rc(bad, 2, out) == 3             # null view field
    assert (out == 7).all()
    assert srv.answer_batch_rc(views, 1, None) == 1          # null output
    assert srv.answer_batch_rc(views, 0, out) == 0           # empty batch is a no-op
    assert (out == 7).all()


@pytest.mark.parametrize("horner", [0, 1, 2])
@pytest.mark.parametrize("matvec_tc", [1, 0])
def test_every_schedule_gives_the_same_responses(batch_env, horner, matvec_tc):
    """Each Horner kernel (one CTA, 4-CTA and 8-CTA clusters) and both
    mat-vec kernels, pinned through ipir_b200_set_schedule, give the
    oracle-checked single answers."""
    c, srv, qs, sts = batch_env
    want = np.stack([srv.answer(q) for q in qs[:4]])
    for n in (1, 4):
        srv.set_schedule(n, matvec_tc=matvec_tc, horner_cluster=horner)
    got = np.stack([srv.answer(q) for q in qs[:2]])
    assert (got == want[:2]).all()
    assert (srv.answer_batch(qs[:4]) == want).all()
    assert (got[0] == c.oracle_answer(qs[0])).all()
    for n in (1, 4):
        srv.set_schedule(n, matvec_tc=1, horner_cluster=1)


@pytest.mark.parametrize("tp_sms", [1, 40, 147])
def test_tensor_pass_beside_matvec(batch_env, tp_sms):
    """The tensor pass on tp_sms SMs from the lane's second stream while the
    mat-vec runs on the others (down to one SM either side) gives the same
    responses as the two one after the other."""
    c, srv, qs, sts = batch_env
    want = np.stack([srv.answer(q) for q in qs])
    for n in (1, 4, 10):
        srv.set_schedule(n, matvec_tc=1, horner_cluster=1, tp_sms=tp_sms)
        assert srv.schedule(n)["tp_sms"] == tp_sms
    assert (srv.answer(qs[0]) == want[0]).all()
    assert (srv.answer_batch(qs[:4]) == want[:4]).all()
    assert (srv.answer_batch(qs) == want).all()
    for n in (1, 4, 10):
        srv.set_schedule(n, matvec_tc=1, horner_cluster=1)
    with pytest.raises(Exception):
        srv.set_schedule(4, matvec_tc=0, horner_cluster=1, tp_sms=8)   # CUDA-core mat-vec: no split


def test_views_contiguous_or_scattered(batch_env):
    """ipir_answer_batch copies each run of query parts that is contiguous in
    host memory at once: a whole batch in one array (one copy), flat queries
    (one copy each) and views whose five parts live in separate arrays (five
    copies each) give the same responses."""
    import inspire_b200 as ib
    c, srv, qs, sts = batch_env
    want = srv.answer_batch(qs)
    n = len(qs)
    rn = ib.response_u64s(srv.params)
    batch = np.ascontiguousarray(np.stack(qs))            # [n][flat] in one array
    views = (ib.IpirQueryView * n)()
    for i in range(n):
        views[i] = ib.query_view_from_flat(srv.params, batch[i])
    out = np.zeros((n, rn), np.uint64)
    assert srv.answer_batch_rc(views, n, out) == 0
    assert (out == want).all()
    R = srv.params["db_rows"]
    blk = 2 * 2 * 2048
    keep = []
    scattered = (ib.IpirQueryView * n)()
    for i in range(n - 1, -1, -1):                         # parts out of order in memory
        q = qs[i]
        parts = [q[:R].copy(), q[R:2 * R].copy(), q[2 * R:2 * R + blk].copy(),
                 q[2 * R + blk:2 * R + 2 * blk].copy(), q[2 * R + 2 * blk:].copy()]
        keep.append(parts)
        v = ib.IpirQueryView()
        for name, a in zip(("lwe_b_limb0", "lwe_b_limb1", "ksk5_b", "kskneg1_b", "rgsw"), parts):
            setattr(v, name, a.ctypes.data_as(ib.u64p))
        scattered[i] = v
    out2 = np.zeros((n, rn), np.uint64)
    assert srv.answer_batch_rc(scattered, n, out2) == 0
    assert (out2 == want).all()


def test_batches_beyond_one_slice(batch_env):
    """Batches of more than 32 queries run as consecutive 32-query slices
    (slice = 32) or as one pipeline (slice = 0); both, through the blocking
    answer, the staged path with stage timing, and the tensor pass beside
    the mat-vec, give every query's single answer (70 = 32 + 32 + 6 and
    40 = 32 + 8 queries, each of the 10 module queries repeated)."""
    import inspire_b200 as ib
    c, srv1, qs, sts = batch_env
    singles = np.stack([srv1.answer(q) for q in qs])
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=70, crs_seed=c.seed)
    try:
        for n in (70, 40):
            batch = [qs[k % len(qs)] for k in range(n)]
            want = np.stack([singles[k % len(qs)] for k in range(n)])
            for sl in (32, 0):
                srv.set_schedule(n, matvec_tc=1, horner_cluster=1, slice=sl)
                assert srv.schedule(n)["slice"] == sl
                assert (srv.answer_batch(batch) == want).all(), (n, sl)
                srv.enable_stage_timing(True)
                assert (srv.answer_batch(batch) == want).all(), (n, sl, "timed")
                st = srv.stage_times()
                srv.enable_stage_timing(False)
                assert all(v > 0 for v in st.values()), st
                srv.set_schedule(n, matvec_tc=1, horner_cluster=1, tp_sms=40, slice=sl)
                assert (srv.answer_batch(batch) == want).all(), (n, sl, "beside")
        with pytest.raises(Exception):
            srv.set_schedule(40, matvec_tc=1, horner_cluster=1, slice=16)
    finally:
        srv.close()
