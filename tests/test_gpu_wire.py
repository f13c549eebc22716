"""Wire formats on the GPU against the reference client library
(src/capi_client.cpp): packed queries unpacked on the device give the same
answers as flat ones; packed and compressed responses are byte-identical to
ipir_response_pack / ipir_response_compress of the flat response, and the
compressed ones decode through the reference's extract_compressed."""
import numpy as np
import pytest

from cases import get_case
from oracle_lib import ref_params

pytestmark = pytest.mark.gpu

IDX = [3, 99999, 524287]


@pytest.fixture(scope="module")
def env():
    import inspire_b200 as ib
    c = get_case("batch")
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=4, crs_seed=c.seed)
    p = ref_params(c.geom, (c.n_entries, c.w), c.seed)
    qs, sts = [], []
    for k, idx in enumerate(IDX):
        q, st = c.query(idx, 8000 + k)
        qs.append(q)
        sts.append(st)
    packed = np.concatenate([c.r.wire(p, "ipir_query_pack", q, "ipir_query_packed_bytes") for q in qs])
    yield c, srv, p, qs, sts, packed
    srv.close()


def test_packed_queries_answer_like_flat(env):
    import inspire_b200 as ib
    c, srv, p, qs, sts, packed = env
    flat = srv.answer_wire(packed, len(qs), ib.RESP_FLAT)
    assert (flat == srv.answer_batch(qs)).all()


def test_packed_and_compressed_responses_match_reference(env):
    import inspire_b200 as ib
    c, srv, p, qs, sts, packed = env
    want = srv.answer_batch(qs)
    got_p = srv.answer_wire(packed, len(qs), ib.RESP_PACKED)
    got_c = srv.answer_wire(packed, len(qs), ib.RESP_COMPRESSED)
    for i, (idx, st) in enumerate(zip(IDX, sts)):
        assert (got_p[i] == c.r.wire(p, "ipir_response_pack", want[i], "ipir_response_packed_bytes")).all(), i
        assert (got_c[i] == c.r.wire(p, "ipir_response_compress", want[i], "ipir_response_compressed_bytes")).all(), i
        assert (st.extract_compressed(got_c[i]) == c.expected_slots(idx)).all(), i


def test_answer_wire_error_codes(env):
    import ctypes as C
    import inspire_b200 as ib
    c, srv, p, qs, sts, packed = env
    L = ib.library_handle()
    out = np.zeros(1 << 20, np.uint8)
    assert L.ipir_b200_answer_wire(srv._h, packed.ctypes.data, 5, 0, out.ctypes.data) == 2   # > max_batch
    assert L.ipir_b200_answer_wire(srv._h, packed.ctypes.data, 1, 7, out.ctypes.data) == 3   # bad format
    assert L.ipir_b200_answer_wire(srv._h, None, 1, 0, out.ctypes.data) == 1
