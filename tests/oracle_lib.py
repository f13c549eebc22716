"""ctypes bindings for the test-only checkers under oracle/.

* ``Oracle``  -- oracle/_build/liboracle.so, the CPU restatement of the
  reference server path (preprocess + answer).
* ``RefLib``  -- oracle/_ref/libinspire_ref.so, the reference's own CPU
  library compiled from its sources (client query/extract and primitives).

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this module.  The product never imports it.
"""
import ctypes as C
import os

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(REPO, "oracle", "_build", "liboracle.so")
REF_SO = os.path.join(REPO, "oracle", "_ref", "libinspire_ref.so")

N = 2048
Q0, Q1 = 94519297, 95293441
QS = (Q0, Q1)
P = 65535
D_EFF = 2
NSTEPS = 1023
PRE_A = 2 * N
PRE_D = 2 * NSTEPS * D_EFF * N
PRE_F = 2 * D_EFF * N

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
u16p = C.POINTER(C.c_uint16)
u8p = C.POINTER(C.c_uint8)


def ptr(a, t):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(t)


class Oracle:
    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(path)
        self.L = L
        L.orc_init.restype = C.c_int
        L.orc_ntt_forward.argtypes = [u64p, C.c_int]
        L.orc_ntt_inverse.argtypes = [u64p, C.c_int]
        L.orc_decomp.argtypes = [u64p, u64p]
        L.orc_expand_seed.argtypes = [u8p, C.c_char_p, C.c_uint64, u64p]
        L.orc_expand_seed.restype = C.c_int
        L.orc_perm_table.argtypes = [C.c_uint32, u32p]
        L.orc_encode.argtypes = [u16p, C.c_size_t, C.c_size_t, C.c_size_t]
        L.orc_crs_polys.argtypes = [u8p, C.c_size_t, u64p]
        L.orc_a_side.argtypes = [u16p, C.c_size_t, C.c_size_t, C.c_size_t, u64p, u64p]
        L.orc_ring_embed_literal.argtypes = [u64p, u32p, C.c_size_t, u64p]
        L.orc_ring_embed_fast.argtypes = [u64p, u64p]
        L.orc_expand_ksk.argtypes = [u8p, u64p, u64p, u64p]
        L.orc_expand_ksk.restype = C.c_int
        L.orc_collapse_group.argtypes = [u64p, u64p, u64p, u64p, u32p, u32p, u32p, u32p]
        L.orc_preprocess.argtypes = [u8p, u16p, C.c_size_t, C.c_size_t, C.c_size_t,
                                     C.c_size_t, C.c_size_t, C.c_int, u32p, u32p, u32p, u32p]
        L.orc_preprocess.restype = C.c_int
        L.orc_matvec.argtypes = [u16p, C.c_size_t, C.c_size_t, u64p, C.c_size_t, C.c_size_t, u64p]
        L.orc_pack_group.argtypes = [u64p, C.c_size_t, C.c_size_t, u32p, u32p, u32p, u64p, u64p, u64p]
        L.orc_ext_prod.argtypes = [u64p, u64p, u64p]
        L.orc_horner.argtypes = [u64p, u64p, C.c_size_t, u64p]
        L.orc_answer.argtypes = [u16p, C.c_size_t, C.c_size_t, C.c_size_t, u32p, u32p, u32p, u32p,
                                 u64p, u64p]
        L.orc_answer.restype = C.c_int
        L.orc_fill_db.argtypes = [u16p, C.c_size_t, C.c_uint64]
        L.orc_fill_u32_mod.argtypes = [u32p, C.c_size_t, C.c_uint64, C.c_uint32]
        L.orc_num_threads.restype = C.c_int
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_init()

    # primitives -----------------------------------------------------
    def ntt_forward(self, a, limb):
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        self.L.orc_ntt_forward(ptr(a, u64p), limb)
        return a

    def ntt_inverse(self, a, limb):
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        self.L.orc_ntt_inverse(ptr(a, u64p), limb)
        return a

    def decomp(self, f):
        f = np.ascontiguousarray(f, dtype=np.uint64)
        out = np.zeros(D_EFF * 2 * N, np.uint64)
        self.L.orc_decomp(ptr(f, u64p), ptr(out, u64p))
        return out

    def expand_seed(self, seed, domain, index):
        s = np.frombuffer(bytes(seed), np.uint8).copy()
        out = np.zeros(2 * N, np.uint64)
        rc = self.L.orc_expand_seed(ptr(s, u8p), domain.encode(), index, ptr(out, u64p))
        assert rc == 0
        return out

    def perm_table(self, t):
        out = np.zeros(N, np.uint32)
        self.L.orc_perm_table(t, ptr(out, u32p))
        return out

    def encode(self, db, rows, cols, D):
        db = np.ascontiguousarray(db, dtype=np.uint16).copy()
        self.L.orc_encode(ptr(db, u16p), rows, cols, D)
        return db

    def fill_db(self, count, seed):
        db = np.empty(count, np.uint16)
        self.L.orc_fill_db(ptr(db, u16p), count, seed)
        return db

    def fill_u32_mod(self, count, seed, q):
        out = np.empty(count, np.uint32)
        self.L.orc_fill_u32_mod(ptr(out, u32p), count, seed, q)
        return out

    def preprocess(self, seed, db, rows, cols, D, group_lo=0, group_hi=None, encode=True):
        G = cols // N
        group_hi = G if group_hi is None else group_hi
        ng = group_hi - group_lo
        db = np.ascontiguousarray(db, dtype=np.uint16).copy()
        s = np.frombuffer(bytes(seed), np.uint8).copy()
        pa = np.zeros(ng * PRE_A, np.uint32)
        pdp = np.zeros(ng * PRE_D, np.uint32)
        pdm = np.zeros(ng * PRE_D, np.uint32)
        pdf = np.zeros(ng * PRE_F, np.uint32)
        rc = self.L.orc_preprocess(ptr(s, u8p), ptr(db, u16p), rows, cols, D, group_lo, group_hi,
                                   1 if encode else 0, ptr(pa, u32p), ptr(pdp, u32p),
                                   ptr(pdm, u32p), ptr(pdf, u32p))
        assert rc == 0, rc
        return db, (pa, pdp, pdm, pdf)

    def answer(self, db_enc, rows, cols, D, pre, qflat):
        G = cols // N
        ncts = max(1, G // D)
        resp = np.zeros(ncts * 4 * N, np.uint64)
        pa, pdp, pdm, pdf = pre
        q = np.ascontiguousarray(qflat, dtype=np.uint64)
        rc = self.L.orc_answer(ptr(db_enc, u16p), rows, cols, D, ptr(pa, u32p), ptr(pdp, u32p),
                               ptr(pdm, u32p), ptr(pdf, u32p), ptr(q, u64p), ptr(resp, u64p))
        assert rc == 0
        return resp

    def matvec(self, db, rows, cols, b, col_lo=0, col_hi=None):
        col_hi = cols if col_hi is None else col_hi
        out = np.zeros(2 * cols, np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        self.L.orc_matvec(ptr(db, u16p), rows, cols, ptr(b, u64p), col_lo, col_hi, ptr(out, u64p))
        return out

    def ext_prod(self, rgsw, ct):
        out = np.zeros(4 * N, np.uint64)
        self.L.orc_ext_prod(ptr(np.ascontiguousarray(rgsw, np.uint64), u64p),
                            ptr(np.ascontiguousarray(ct, np.uint64), u64p), ptr(out, u64p))
        return out

    def horner(self, rgsw, packed, L):
        out = np.zeros(4 * N, np.uint64)
        self.L.orc_horner(ptr(np.ascontiguousarray(rgsw, np.uint64), u64p),
                          ptr(np.ascontiguousarray(packed, np.uint64), u64p), L, ptr(out, u64p))
        return out


class RefParams(C.Structure):
    """ipir_params of the reference's capi.h (src/capi.h:27-38)."""
    _fields_ = [("n_entries", C.c_size_t), ("entry_bytes", C.c_size_t), ("db_rows", C.c_size_t),
                ("db_cols", C.c_size_t), ("n_packed", C.c_size_t), ("interp_d", C.c_size_t),
                ("num_cts", C.c_size_t), ("ring_n", C.c_size_t), ("d_eff", C.c_size_t),
                ("seed", C.c_uint8 * 64)]


def ref_params(geom, entry_bytes_and_entries, crs_seed):
    """RefParams from a setup() geometry [n_entries, w, R, C, G, D, num_cts]."""
    p = RefParams()
    p.n_entries, p.entry_bytes = entry_bytes_and_entries
    p.db_rows, p.db_cols, p.n_packed, p.interp_d, p.num_cts = geom[2], geom[3], geom[4], geom[5], geom[6]
    p.ring_n, p.d_eff = N, 2
    p.seed[:] = list(bytes(crs_seed))
    return p


class RefLib:
    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        L = C.CDLL(path)
        self.L = L
        L.refh_setup.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, u64p]
        L.refh_setup.restype = C.c_int
        L.refh_query.argtypes = [u64p, u8p, C.c_uint64, C.c_uint64, u64p]
        L.refh_query.restype = C.c_void_p
        L.refh_extract.argtypes = [C.c_void_p, u64p, u16p, u64p]
        L.refh_extract.restype = C.c_int
        L.refh_decrypt.argtypes = [C.c_void_p, u64p, u64p]
        L.refh_state_free.argtypes = [C.c_void_p]
        L.refh_ntt_forward.argtypes = [u64p, C.c_int]
        L.refh_ntt_inverse.argtypes = [u64p, C.c_int]
        L.refh_ntt_tables.argtypes = [C.c_int, u64p, u64p, u64p, u64p]
        L.refh_decomp.argtypes = [u64p, u64p]
        L.refh_expand_seed.argtypes = [u8p, C.c_char_p, C.c_uint64, u64p]
        L.refh_automorphism_ntt.argtypes = [u64p, C.c_uint64, u64p]
        L.refh_ext_prod.argtypes = [u64p, u64p, u64p]
        L.refh_horner_eval.argtypes = [u64p, u64p, C.c_uint64, u64p]
        L.refh_extract_compressed.argtypes = [C.c_void_p, u8p, u16p, u64p]
        L.refh_extract_compressed.restype = C.c_int
        # the reference client library's wire codecs (src/capi_client.cpp)
        for fn in ("ipir_query_packed_bytes", "ipir_response_packed_bytes", "ipir_response_compressed_bytes"):
            getattr(L, fn).argtypes = [C.POINTER(RefParams)]
            getattr(L, fn).restype = C.c_size_t
        for fn in ("ipir_query_pack", "ipir_response_pack", "ipir_response_compress"):
            getattr(L, fn).argtypes = [C.POINTER(RefParams), u64p, u8p]
            getattr(L, fn).restype = C.c_int
        L.ipir_query_unpack.argtypes = [C.POINTER(RefParams), u8p, u64p]
        L.ipir_query_unpack.restype = C.c_int

    def setup(self, n_entries, w, db_rows=0):
        g = np.zeros(7, np.uint64)
        rc = self.L.refh_setup(n_entries, w, db_rows, ptr(g, u64p))
        if rc != 0:
            raise ValueError("setup() rejected the geometry")
        return [int(x) for x in g]

    def wire(self, params, fn, flat, nbytes_fn):
        """Run one of the reference's packers on a flat u64 array."""
        nb = getattr(self.L, nbytes_fn)(C.byref(params))
        out = np.zeros(nb, np.uint8)
        flat = np.ascontiguousarray(flat, np.uint64)
        assert getattr(self.L, fn)(C.byref(params), ptr(flat, u64p), ptr(out, u8p)) == 0
        return out

    def query(self, geom, crs_seed, idx, rng_seed):
        g = np.array(geom, np.uint64)
        s = np.frombuffer(bytes(crs_seed), np.uint8).copy()
        flat = np.zeros(query_u64s(geom), np.uint64)
        st = self.L.refh_query(ptr(g, u64p), ptr(s, u8p), idx, rng_seed, ptr(flat, u64p))
        assert st
        return flat, RefState(self, st)

    def ntt_forward(self, a, limb):
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        self.L.refh_ntt_forward(ptr(a, u64p), limb)
        return a

    def ntt_inverse(self, a, limb):
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        self.L.refh_ntt_inverse(ptr(a, u64p), limb)
        return a

    def tables(self, limb):
        fwd = np.zeros(N, np.uint64)
        inv = np.zeros(N, np.uint64)
        inv_n = np.zeros(1, np.uint64)
        psi = np.zeros(1, np.uint64)
        self.L.refh_ntt_tables(limb, ptr(fwd, u64p), ptr(inv, u64p), ptr(inv_n, u64p), ptr(psi, u64p))
        return fwd, inv, int(inv_n[0]), int(psi[0])

    def decomp(self, f):
        out = np.zeros(D_EFF * 2 * N, np.uint64)
        self.L.refh_decomp(ptr(np.ascontiguousarray(f, np.uint64), u64p), ptr(out, u64p))
        return out

    def expand_seed(self, seed, domain, index):
        s = np.frombuffer(bytes(seed), np.uint8).copy()
        out = np.zeros(2 * N, np.uint64)
        self.L.refh_expand_seed(ptr(s, u8p), domain.encode(), index, ptr(out, u64p))
        return out

    def automorphism_ntt(self, f, k):
        out = np.zeros(2 * N, np.uint64)
        self.L.refh_automorphism_ntt(ptr(np.ascontiguousarray(f, np.uint64), u64p), k, ptr(out, u64p))
        return out

    def ext_prod(self, rgsw, ct):
        out = np.zeros(4 * N, np.uint64)
        self.L.refh_ext_prod(ptr(np.ascontiguousarray(rgsw, np.uint64), u64p),
                             ptr(np.ascontiguousarray(ct, np.uint64), u64p), ptr(out, u64p))
        return out

    def horner(self, rgsw, cts, L):
        out = np.zeros(4 * N, np.uint64)
        self.L.refh_horner_eval(ptr(np.ascontiguousarray(rgsw, np.uint64), u64p),
                                ptr(np.ascontiguousarray(cts, np.uint64), u64p), L, ptr(out, u64p))
        return out


class RefState:
    def __init__(self, lib, handle):
        self.lib = lib
        self.h = handle

    def extract(self, resp):
        slots = np.zeros(N, np.uint16)
        n = np.zeros(1, np.uint64)
        resp = np.ascontiguousarray(resp, np.uint64)
        rc = self.lib.L.refh_extract(self.h, ptr(resp, u64p), ptr(slots, u16p), ptr(n, u64p))
        assert rc == 0
        return slots[: int(n[0])]

    def extract_compressed(self, data):
        slots = np.zeros(N, np.uint16)
        n = np.zeros(1, np.uint64)
        data = np.ascontiguousarray(data, np.uint8)
        rc = self.lib.L.refh_extract_compressed(self.h, ptr(data, u8p), ptr(slots, u16p), ptr(n, u64p))
        assert rc == 0
        return slots[: int(n[0])]

    def decrypt(self, resp):
        m = np.zeros(N, np.uint64)
        resp = np.ascontiguousarray(resp, np.uint64)
        self.lib.L.refh_decrypt(self.h, ptr(resp, u64p), ptr(m, u64p))
        return m

    def __del__(self):
        try:
            self.lib.L.refh_state_free(self.h)
        except Exception:
            pass


def query_u64s(geom):
    return 2 * geom[2] + 6 * D_EFF * 2 * N


def crs_seed_from(s):
    """64-byte CRS seed: mt19937_64(s)() & 0xFF per byte (the convention the
    parity cases use; the reference draws it from std::random_device)."""
    return bytes(int(x) & 0xFF for x in mt19937_64(s, 64))


def mt19937_64(seed, n):
    """std::mt19937_64 outputs (for seeds shared with the C++ harness)."""
    NN, MM = 312, 156
    MATRIX_A = 0xB5026F5AA96619E9
    UM, LM = 0xFFFFFFFF80000000, 0x7FFFFFFF
    mt = [0] * NN
    mt[0] = seed & 0xFFFFFFFFFFFFFFFF
    for i in range(1, NN):
        mt[i] = (6364136223846793005 * (mt[i - 1] ^ (mt[i - 1] >> 62)) + i) & 0xFFFFFFFFFFFFFFFF
    idx = NN
    out = []
    for _ in range(n):
        if idx >= NN:
            for i in range(NN):
                x = (mt[i] & UM) | (mt[(i + 1) % NN] & LM)
                xa = x >> 1
                if x & 1:
                    xa ^= MATRIX_A
                mt[i] = mt[(i + MM) % NN] ^ xa
            idx = 0
        y = mt[idx]
        idx += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFA0000000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        out.append(y & 0xFFFFFFFFFFFFFFFF)
    return out


def entry_slots(geom, db, idx):
    """The cpe DB slots of entry idx (row-major db[row*cols+col]), as the
    reference tests check them (tests/test_e2e_gpu.cu:95-104)."""
    n_entries, w, rows, cols = geom[0], geom[1], geom[2], geom[3]
    cpe = (w * 8 + 14) // 15
    i_star = idx % rows
    col = (idx // rows) * cpe
    return np.array([db[i_star * cols + col + c] % P for c in range(cpe)], np.uint16)
