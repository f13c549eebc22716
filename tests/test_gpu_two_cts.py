"""Two response ciphertexts per query: 512 packing groups > D = 256 on a
2048-row DB (the structure of the 64 GB geometry), 34 GB of precomputed
tensors.  Each ciphertext's Horner chain covers 256 groups; entries in
both halves are retrieved.  Parity is size-independent (the oracle is too
slow here): batch == singles, extract() recovers every entry, the wire
formats are byte-identical to the reference client library's and the
compressed responses decode."""
import numpy as np
import pytest

from cases import get_case
from oracle_lib import ref_params

pytestmark = pytest.mark.gpu

IDX = [5, 2048 * 8192 + 7, 33554431]   # ciphertext 0, ciphertext 1, last entry


@pytest.fixture(scope="module")
def env():
    import inspire_b200 as ib
    c = get_case("g512")
    assert c.G == 512 and c.ncts == 2
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=3, crs_seed=c.seed)
    qs, sts = [], []
    for k, idx in enumerate(IDX):
        q, st = c.query(idx, 9000 + k)
        qs.append(q)
        sts.append(st)
    yield c, srv, qs, sts
    srv.close()


def test_two_ciphertexts_batch_singles_extract(env):
    c, srv, qs, sts = env
    singles = np.stack([srv.answer(q) for q in qs])
    assert singles.shape[1] == 2 * 4 * 2048
    assert (srv.answer_batch(qs) == singles).all()
    for i, st in enumerate(sts):
        assert (st.extract(singles[i]) == c.expected_slots(IDX[i])).all(), i


def test_two_ciphertexts_wire_formats(env):
    import inspire_b200 as ib
    c, srv, qs, sts = env
    p = ref_params(c.geom, (c.n_entries, c.w), c.seed)
    packed = np.concatenate([c.r.wire(p, "ipir_query_pack", q, "ipir_query_packed_bytes") for q in qs])
    want = srv.answer_batch(qs)
    got_p = srv.answer_wire(packed, len(qs), ib.RESP_PACKED)
    got_c = srv.answer_wire(packed, len(qs), ib.RESP_COMPRESSED)
    for i, (idx, st) in enumerate(zip(IDX, sts)):
        assert (got_p[i] == c.r.wire(p, "ipir_response_pack", want[i], "ipir_response_packed_bytes")).all(), i
        assert (got_c[i] == c.r.wire(p, "ipir_response_compress", want[i], "ipir_response_compressed_bytes")).all(), i
        assert (st.extract_compressed(got_c[i]) == c.expected_slots(idx)).all(), i


def test_two_ciphertexts_chunked_horner(env):
    """The Horner chains trailing the DB pass in chunks with two response
    ciphertexts: each chunk is the same range of chain positions in both
    (one mat-vec launch over the two column ranges), both chains resume
    from memory; every chunking and both cluster kernels give the
    unchunked responses."""
    c, srv, qs, sts = env
    for n in (1, 3):
        srv.set_schedule(n, matvec_tc=1, horner_cluster=1)
    want = srv.answer_batch(qs)
    assert (srv.answer(qs[1]) == want[1]).all()
    for hc in (1, 2):
        for k in (2, 3, 8):
            for n in (1, 3):
                srv.set_schedule(n, matvec_tc=1, horner_cluster=hc, hchunks=k)
            assert (srv.answer_batch(qs) == want).all(), (hc, k)
            assert (srv.answer(qs[1]) == want[1]).all(), (hc, k)
    for i, st in enumerate(sts):
        assert (st.extract(want[i]) == c.expected_slots(IDX[i])).all(), i
    for n in (1, 3):
        srv.set_schedule(n, matvec_tc=1, horner_cluster=1)
