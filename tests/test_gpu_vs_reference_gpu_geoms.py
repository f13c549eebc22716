"""Bit-exact parity with the reference's own GPU server at the benchmark
geometries (the reference library is its five .cu files compiled for sm_100a
by oracle/Makefile into oracle/_ref).

For each geometry both servers are built from the same DB and CRS seed.  64
reference-client queries are made on uniform indices (mt19937_64(seed) mod
N_entries); the last 8 repeat the first 8 indices with fresh client keys,
so a batch holds the same index twice (reference tests/test_gpu_batch.cu:51-56:
no dedup by index).  The reference answers all 64 in one ipir_answer_batch.
This server answers them at B = 1 (the first 4, one call each), B = 8, 32
and 64, after autotuning (the schedules bench.py times), and every response
must equal the reference's u64 for u64; extract() must then return each
queried entry (reference tests/test_e2e_gpu.cu:95-104).

Geometries (w = 30 / 960 stand in for 32 / 1024, which setup() rejects,
with the same DB bytes):
  cfg2    setup(2^25, 30)       R 32768, C 16384,  G 8,   1.07 GB
  g128    setup(2^23, 120, 2048) R 2048, C 262144, G 128, 1.07 GB
  cfg5b   setup(2^22, 960)      R 32768, C 65536,  G 32,  4.29 GB (two-pass encode)
  cfg3    setup(2^29, 30)       R 32768, C 262144, G 128, 17.18 GB (the headline)
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle_lib import Oracle, RefLib, crs_seed_from, entry_slots, mt19937_64

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

REF_GPU = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libinspire_ref_gpu.so")

GEOMS = {
    # name: (n_entries, w, db_rows_arg, crs seed, db seed, index seed)
    "cfg2": (1 << 25, 30, 0, 1, 0, 3),
    "g128": (1 << 23, 120, 2048, 3, 5, 11),
    "cfg5b": (1 << 22, 960, 0, 9, 1, 6),
    "cfg3": (1 << 29, 30, 0, 1, 0, 4),
}
NQ = 64
NDUP = 8


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


def indices(n_entries, seed):
    base = [x % n_entries for x in mt19937_64(seed, NQ - NDUP)]
    return base + base[:NDUP]


@pytest.mark.parametrize("name", list(GEOMS))
def test_geometry_bit_exact_vs_reference_gpu(refgpu, name):
    import inspire_b200 as ib
    n_entries, w, rows_arg, crs, db_seed, idx_seed = GEOMS[name]
    ref = RefLib()
    geom = ref.setup(n_entries, w, rows_arg)
    R, Cc = geom[2], geom[3]
    seed = crs_seed_from(crs)
    db = Oracle().fill_db(R * Cc, db_seed)
    idx = indices(n_entries, idx_seed)

    seed_arr = np.frombuffer(seed, np.uint8).copy()
    p = ib.IpirParams()
    h = refgpu.ipir_server_create(n_entries, w, rows_arg, NQ, db.ctypes.data, seed_arr.ctypes.data, C.byref(p))
    assert h, "reference ipir_server_create failed"
    try:
        qs, sts = [], []
        for k, i in enumerate(idx):
            q, st = ref.query(geom, seed, i, 7000 + k)   # fresh keys per query, duplicates included
            qs.append(np.ascontiguousarray(q, np.uint64))
            sts.append(st)
        assert (qs[0] != qs[NQ - NDUP]).any(), "a repeated index must come with fresh keys"
        views = (ib.IpirQueryView * NQ)()
        for k, q in enumerate(qs):
            views[k] = ib.query_view_from_flat(p.as_dict(), q)
        rn = p.num_cts * 4 * 2048
        want = np.zeros((NQ, rn), np.uint64)
        assert refgpu.ipir_answer_batch(h, views, NQ, want.ctypes.data) == 0
    finally:
        refgpu.ipir_server_destroy(h)

    srv = ib.Server(n_entries, w, db, db_rows=rows_arg, max_batch=NQ, crs_seed=seed)
    try:
        assert srv.params["db_cols"] == Cc and srv.params["num_cts"] == p.num_cts
        srv.autotune()
        for k in range(4):
            got = srv.answer(qs[k])
            assert np.array_equal(got, want[k]), f"{name}: B=1 query {k} differs from the reference GPU server"
        for b in (8, 32, NQ):
            got = srv.answer_batch(qs[:b])
            bad = [k for k in range(b) if not np.array_equal(got[k], want[k])]
            assert not bad, f"{name}: B={b} responses {bad[:8]} differ from the reference GPU server"
        # the Horner chain trailing the DB pass in chunks, whatever the
        # autotuner picked: 8 chunks with each cluster Horner kernel
        for hc in (1, 2):
            for b in (1, 8):
                srv.set_schedule(b, matvec_tc=1, horner_cluster=hc, hchunks=8)
            assert np.array_equal(srv.answer(qs[0]), want[0]), f"{name}: chunked B=1 (Horner kernel {hc})"
            got = srv.answer_batch(qs[:8])
            bad = [k for k in range(8) if not np.array_equal(got[k], want[k])]
            assert not bad, f"{name}: chunked B=8 (Horner kernel {hc}) responses {bad} differ"
    finally:
        srv.close()
    for k, st in enumerate(sts):
        assert (st.extract(want[k]) == entry_slots(geom, db, idx[k])).all(), (name, k)
