"""Responses bit-identical to the reference's own GPU server (its five .cu
files compiled for sm_100a by oracle/Makefile into oracle/_ref): same DB,
same CRS seed, same client queries, both through the same C ABI
(ipir_server_create / ipir_answer_batch)."""
import ctypes as C
import os

import numpy as np
import pytest

from cases import get_case

pytestmark = pytest.mark.gpu

REF_GPU = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libinspire_ref_gpu.so")


@pytest.fixture(scope="module")
def refgpu():
    import inspire_b200 as ib
    if not os.path.exists(REF_GPU):
        pytest.skip("reference GPU library not built (needs the reference sources)")
    L = C.CDLL(REF_GPU)  # RTLD_LOCAL: its ipir_* names stay separate from ours
    L.ipir_server_create.restype = C.c_void_p
    L.ipir_server_create.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p,
                                     C.POINTER(ib.IpirParams)]
    L.ipir_answer_batch.argtypes = [C.c_void_p, C.POINTER(ib.IpirQueryView), C.c_size_t, C.c_void_p]
    L.ipir_answer_batch.restype = C.c_int
    L.ipir_server_destroy.argtypes = [C.c_void_p]
    return L


@pytest.mark.parametrize("name,idx", [("small", [0, 200, 255]), ("medium", [7, 131072, 262143]),
                                      ("batch", [1, 300000, 524287])])
def test_responses_equal_reference_gpu(refgpu, name, idx):
    import inspire_b200 as ib
    c = get_case(name)
    seed = np.frombuffer(bytes(c.seed), np.uint8).copy()
    db = np.ascontiguousarray(c.db, np.uint16)
    p = ib.IpirParams()
    h = refgpu.ipir_server_create(c.n_entries, c.w, 2048, len(idx), db.ctypes.data, seed.ctypes.data, C.byref(p))
    assert h, "reference ipir_server_create failed"
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=len(idx), crs_seed=c.seed)
    try:
        qs, sts = [], []
        for k, i in enumerate(idx):
            q, st = c.query(i, 4000 + k)
            qs.append(np.ascontiguousarray(q, np.uint64))
            sts.append(st)
        views = (ib.IpirQueryView * len(qs))()
        for k, q in enumerate(qs):
            views[k] = ib.query_view_from_flat(srv.params, q)
        want = np.zeros((len(qs), ib.response_u64s(srv.params)), np.uint64)
        assert refgpu.ipir_answer_batch(h, views, len(qs), want.ctypes.data) == 0
        got = srv.answer_batch(qs)
        assert (got == want).all()
        for k, st in enumerate(sts):
            assert (st.extract(got[k]) == c.expected_slots(idx[k])).all(), k
    finally:
        srv.close()
        refgpu.ipir_server_destroy(h)
