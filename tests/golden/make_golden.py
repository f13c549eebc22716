"""Generates the golden parity fixtures in this folder (``*.npz``).

Each fixture is one client query answered by the reference's own GPU server
(oracle/_ref/libinspire_ref_gpu.so, compiled for sm_100a from the
reference's sources by ``make -C oracle ref_gpu``) through its C ABI
(``ipir_server_create`` / ``ipir_answer_batch``, src/capi.h:76-89).  It
therefore runs on a B200 with the reference build present; the tests that
read the fixtures need neither.

Fixture fields: the geometry (``n_entries``, ``w``, ``db_rows``, ``geom`` =
[n_entries, w, R, C, G, D, num_cts]); ``crs`` and ``db_seed``, from which the
tests rebuild the inputs (CRS seed byte i = mt19937_64(crs) output i & 0xFF;
DB value k = splitmix64(db_seed ^ k) mod 65535, row-major) and
``db_sha256`` of that DB; the queried ``idx``; ``query_packed``, the
reference client's query (mt19937_64(``rng``)) in its 53-bit packed wire
format (``ipir_query_pack``); the reference server's response packed
(``ipir_response_pack``, ``resp_packed``) and compressed
(``ipir_response_compress``, ``resp_compressed``); and ``slots``, the DB
entry the client's ``extract()`` returns.

Before writing, every response is checked against the oracle (bit-exact)
and decoded by the client's ``extract()`` and ``extract_compressed()``.

    python tests/golden/make_golden.py [outdir]      # default: this folder
"""
import ctypes as C
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(REPO, "tests"), os.path.join(REPO, "oracle")]

from cases import Case  # noqa: E402
from oracle_lib import RefParams, ref_params  # noqa: E402
import wire  # noqa: E402

REF_GPU = os.path.join(REPO, "oracle", "_ref", "libinspire_ref_gpu.so")
u64p = C.POINTER(C.c_uint64)

# name: (n_entries, w, db_rows, crs, db_seed, idx, rng)
FIXTURES = {
    "small_g1": (256, 120, 2048, 1, 0, 200, 4100),         # G = 1: no Horner
    "medium_g4": (262144, 120, 2048, 1, 0, 131072, 4101),  # G = 4: Horner over 4 packed cts
}


class QueryView(C.Structure):
    """ipir_query_view (src/capi.h:55-61)."""
    _fields_ = [("lwe_b_limb0", u64p), ("lwe_b_limb1", u64p), ("ksk5_b", u64p),
                ("kskneg1_b", u64p), ("rgsw", u64p)]


def view_of(flat, R):
    blk = 2 * 2 * wire.N
    base = flat.ctypes.data
    v = QueryView()
    for name, off in (("lwe_b_limb0", 0), ("lwe_b_limb1", R), ("ksk5_b", 2 * R), ("kskneg1_b", 2 * R + blk),
                      ("rgsw", 2 * R + 2 * blk)):
        setattr(v, name, C.cast(base + 8 * off, u64p))
    return v


def reference_gpu_answer(L, c, q):
    seed = np.frombuffer(bytes(c.seed), np.uint8).copy()
    db = np.ascontiguousarray(c.db, np.uint16)
    p = RefParams()
    h = L.ipir_server_create(c.n_entries, c.w, c.db_rows_arg, 1, db.ctypes.data, seed.ctypes.data, C.byref(p))
    if not h:
        raise RuntimeError("reference ipir_server_create failed")
    try:
        q = np.ascontiguousarray(q, np.uint64)
        views = (QueryView * 1)(view_of(q, c.R))
        out = np.zeros(c.ncts * 4 * wire.N, np.uint64)
        rc = L.ipir_answer_batch(h, views, 1, out.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"reference ipir_answer_batch returned {rc}")
        return out
    finally:
        L.ipir_server_destroy(h)


def main(outdir):
    L = C.CDLL(REF_GPU)
    L.ipir_server_create.restype = C.c_void_p
    L.ipir_server_create.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p,
                                     C.POINTER(RefParams)]
    L.ipir_answer_batch.argtypes = [C.c_void_p, C.POINTER(QueryView), C.c_size_t, C.c_void_p]
    L.ipir_answer_batch.restype = C.c_int
    L.ipir_server_destroy.argtypes = [C.c_void_p]
    os.makedirs(outdir, exist_ok=True)
    for name, (n_entries, w, db_rows, crs, db_seed, idx, rng) in FIXTURES.items():
        c = Case(n_entries, w, db_rows, crs=crs, db_seed=db_seed)
        q, st = c.query(idx, rng)
        resp = reference_gpu_answer(L, c, q)
        assert (resp == c.oracle_answer(q)).all(), f"{name}: reference GPU server and oracle differ"
        slots = c.expected_slots(idx)
        assert (st.extract(resp) == slots).all(), f"{name}: extract() does not return the entry"
        p = ref_params(c.geom, (n_entries, w), c.seed)
        qp = c.r.wire(p, "ipir_query_pack", q, "ipir_query_packed_bytes")
        rp = c.r.wire(p, "ipir_response_pack", resp, "ipir_response_packed_bytes")
        rcm = c.r.wire(p, "ipir_response_compress", resp, "ipir_response_compressed_bytes")
        assert (st.extract_compressed(rcm) == slots).all(), f"{name}: extract_compressed() differs"
        assert (wire.unpack_query(qp, c.R) == q).all() and (wire.unpack_response(rp, c.ncts) == resp).all()
        path = os.path.join(outdir, name + ".npz")
        np.savez_compressed(path, n_entries=n_entries, w=w, db_rows=db_rows, geom=np.array(c.geom, np.uint64),
                            crs=crs, db_seed=db_seed, idx=idx, rng=rng,
                            db_sha256=hashlib.sha256(np.ascontiguousarray(c.db, np.uint16).tobytes()).hexdigest(),
                            query_packed=qp, resp_packed=rp, resp_compressed=rcm, slots=slots)
        print(f"{name}: {os.path.getsize(path)} bytes, geometry {c.geom}, entry {idx}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE)
