"""Python host binding of the B200-native InsPIRe PIR server.

A thin ctypes layer over ``libinspire_b200.so`` (the C ABI declared in
``include/inspire_b200.h``), mirroring the reference's server C ABI
(SoraSuegami/InsPIRe-GPU src/capi.h:23-91): ``ipir_server_create``,
``ipir_server_caps``, ``ipir_answer_batch``, ``ipir_server_destroy``, with the
same flat layouts:

* query   ``[b0: db_rows][b1: db_rows][ksk5: blk][kskneg1: blk][rgsw: 4 blk]``
  u64, ``blk = d_eff * 2 * ring_n`` (``ipir_query_view_from_flat``,
  reference src/capi.h:109-116);
* response ``[ct][a|b][limb][coeff]`` u64 per query, NTT form.

There is no CPU fallback: every computation runs in the CUDA library, and
importing this module fails loudly when the library is missing.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libinspire_b200.so")

RING_N = 2048
D_EFF = 2
Q0, Q1 = 94519297, 95293441
P = 65535
NSTEPS = 1023

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `make -C inspire-gpu_b200` "
                      "(there is no CPU fallback)")
_L = C.CDLL(LIB_PATH)

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
u16p = C.POINTER(C.c_uint16)
u8p = C.POINTER(C.c_uint8)


class IpirParams(C.Structure):
    _fields_ = [("n_entries", C.c_size_t), ("entry_bytes", C.c_size_t), ("db_rows", C.c_size_t),
                ("db_cols", C.c_size_t), ("n_packed", C.c_size_t), ("interp_d", C.c_size_t),
                ("num_cts", C.c_size_t), ("ring_n", C.c_size_t), ("d_eff", C.c_size_t),
                ("seed", C.c_uint8 * 64)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f != "seed"}
        d["seed"] = bytes(self.seed)
        return d


class IpirCaps(C.Structure):
    _fields_ = [("max_batch", C.c_size_t), ("resident_bytes", C.c_size_t),
                ("device_free_bytes", C.c_size_t), ("num_cts", C.c_size_t)]


class IpirQueryView(C.Structure):
    _fields_ = [("lwe_b_limb0", u64p), ("lwe_b_limb1", u64p), ("ksk5_b", u64p),
                ("kskneg1_b", u64p), ("rgsw", u64p)]


_L.ipir_server_create.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, u16p, u8p,
                                  C.POINTER(IpirParams)]
_L.ipir_server_create.restype = C.c_void_p
_L.ipir_server_caps.argtypes = [C.c_void_p, C.POINTER(IpirCaps)]
_L.ipir_server_caps.restype = None
_L.ipir_answer_batch.argtypes = [C.c_void_p, C.POINTER(IpirQueryView), C.c_size_t, u64p]
_L.ipir_answer_batch.restype = C.c_int
_L.ipir_server_destroy.argtypes = [C.c_void_p]
_L.ipir_server_destroy.restype = None
_L.ipir_b200_last_error.restype = C.c_char_p
_L.ipir_b200_setup.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t, C.POINTER(IpirParams)]
_L.ipir_b200_setup.restype = C.c_int
_L.ipir_b200_set_stream.argtypes = [C.c_void_p, C.c_void_p]
_L.ipir_b200_stage_queries.argtypes = [C.c_void_p, C.POINTER(IpirQueryView), C.c_size_t]
_L.ipir_b200_run.argtypes = [C.c_void_p, C.c_size_t]
_L.ipir_b200_fetch_responses.argtypes = [C.c_void_p, C.c_size_t, u64p]
_L.ipir_b200_sync.argtypes = [C.c_void_p]
_L.ipir_b200_enable_stage_timing.argtypes = [C.c_void_p, C.c_int]
_L.ipir_b200_stage_times.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_size_t]
_L.ipir_b200_export_precomp.argtypes = [C.c_void_p, C.c_size_t, u32p, u32p, u32p, u32p]
_L.ipir_b200_export_db.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, u16p]
_L.ipir_b200_ntt.argtypes = [u32p, C.c_size_t, C.c_int, C.c_int]
_L.ipir_b200_decomp.argtypes = [u32p, u32p, C.c_size_t]
_L.ipir_b200_shake256.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t]
_L.ipir_b200_expand_seed.argtypes = [u8p, C.c_char_p, C.c_uint64, u32p]
_L.ipir_b200_fill_db.argtypes = [u16p, C.c_size_t, C.c_uint64]
_L.ipir_b200_matvec.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                                C.c_void_p, C.c_int]
_L.ipir_b200_matvec_noalloc.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_size_t,
                                        C.c_void_p, C.c_void_p]


class IpirSchedule(C.Structure):
    _fields_ = [("matvec_tc", C.c_int), ("tp_pass", C.c_int), ("horner_cluster", C.c_int), ("tp_sms", C.c_int),
                ("slice", C.c_int), ("hchunks", C.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class IpirServeConfig(C.Structure):
    _fields_ = [("max_batch", C.c_size_t), ("lanes_per_db", C.c_size_t), ("queue_slots", C.c_size_t),
                ("hbm_budget_bytes", C.c_size_t), ("disable_graphs", C.c_int), ("disable_autotune", C.c_int),
                ("overlap_db_passes", C.c_int), ("scan_segments", C.c_int)]


class IpirServeCounters(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("batches", C.c_uint64), ("batched_queries", C.c_uint64), ("max_batch_seen", C.c_uint64),
                ("queued", C.c_size_t), ("free_slots", C.c_size_t), ("max_notice_ms", C.c_double)]


class IpirMatvecOpts(C.Structure):
    _fields_ = [("path", C.c_int), ("queries_per_pass", C.c_int), ("kchunk_rows", C.c_int)]


_L.ipir_b200_matvec_ex.argtypes = [C.c_void_p, C.c_size_t, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p,
                                   C.c_void_p, C.c_int, C.POINTER(IpirMatvecOpts)]
_L.ipir_b200_fill_db_device.argtypes = [C.c_void_p, C.c_size_t, C.c_uint64, C.c_void_p]
_L.ipir_b200_kernel_binary_version.argtypes = [C.POINTER(C.c_int)]
_L.ipir_b200_kernel_binary_version.restype = C.c_int
_L.ipir_b200_autotune.argtypes = [C.c_void_p]
_L.ipir_b200_get_schedule.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(IpirSchedule)]
_L.ipir_b200_launch_count.argtypes = [C.c_void_p, C.POINTER(C.c_ulonglong)]
_L.ipir_b200_set_schedule.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(IpirSchedule)]
_L.ipir_b200_wire_sizes.argtypes = [C.POINTER(IpirParams), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                    C.POINTER(C.c_size_t)]
_L.ipir_b200_answer_wire.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_void_p]
RESP_FLAT, RESP_PACKED, RESP_COMPRESSED = 0, 1, 2
_L.ipir_serve_create.restype = C.c_void_p
_L.ipir_serve_create.argtypes = [C.POINTER(C.c_void_p), C.c_size_t, C.POINTER(IpirServeConfig)]
_L.ipir_serve_submit.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(IpirQueryView), C.POINTER(C.c_uint64)]
_L.ipir_serve_poll.argtypes = [C.c_void_p, C.c_uint64, u64p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
_L.ipir_serve_wait.argtypes = [C.c_void_p, C.c_uint64, C.c_double, u64p, C.POINTER(C.c_double),
                               C.POINTER(C.c_double)]
_L.ipir_serve_stats.argtypes = [C.c_void_p, C.POINTER(IpirServeCounters)]
_L.ipir_serve_db_info.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                  C.POINTER(IpirSchedule), C.c_size_t]
_L.ipir_serve_destroy.argtypes = [C.c_void_p]
_L.ipir_b200_shard_create.restype = C.c_void_p
_L.ipir_b200_shard_create.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t, C.c_size_t, u16p, u8p, C.c_size_t,
                                      C.c_size_t, C.c_void_p]
_L.ipir_b200_shard_export_a.argtypes = [C.c_void_p, u32p]
_L.ipir_b200_shard_export_a.restype = C.c_int
_L.ipir_b200_shard_pack.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
_L.ipir_b200_shard_pack.restype = C.c_int
_L.ipir_b200_shard_destroy.argtypes = [C.c_void_p]
_L.ipir_b200_shard_answer.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, u64p]
_L.ipir_b200_shard_answer.restype = C.c_int
_L.ipir_b200_horner_create.restype = C.c_void_p
_L.ipir_b200_horner_create.argtypes = [C.c_void_p, u32p, C.c_size_t]
_L.ipir_b200_horner_answer.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, u64p, C.c_void_p]
_L.ipir_b200_horner_answer.restype = C.c_int
_L.ipir_b200_horner_destroy.argtypes = [C.c_void_p]
_L.ipir_b200_synth_queries.argtypes = [C.c_size_t, C.c_uint64, C.c_uint64, C.c_size_t, C.c_void_p, C.c_void_p]
_L.ipir_b200_synth_queries.restype = C.c_int
_L.ipir_b200_horner_eval.argtypes = [u64p, u64p, C.c_size_t, u64p, C.c_int]
_L.ipir_b200_horner_eval.restype = C.c_int
_L.ipir_serve_replace_db.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
_L.ipir_b200_save_server.argtypes = [C.c_void_p, C.c_char_p]
_L.ipir_b200_save_server.restype = C.c_int
_L.ipir_b200_load_server.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(IpirParams)]
_L.ipir_b200_load_server.restype = C.c_void_p


class IpirServeBatchRecord(C.Structure):
    _fields_ = [("t_issue_s", C.c_double), ("issue_ms", C.c_float), ("device_ms", C.c_float),
                ("notice_ms", C.c_float), ("db", C.c_uint16), ("lane", C.c_uint16), ("count", C.c_uint32),
                ("failed", C.c_uint32)]


_L.ipir_serve_trace.restype = C.c_size_t
_L.ipir_serve_trace.argtypes = [C.c_void_p, C.POINTER(IpirServeBatchRecord), C.c_size_t]

EXPORTED = [
    "ipir_server_create", "ipir_server_caps", "ipir_answer_batch", "ipir_server_destroy",
    "ipir_b200_last_error", "ipir_b200_setup", "ipir_b200_set_stream", "ipir_b200_stage_queries",
    "ipir_b200_run", "ipir_b200_fetch_responses", "ipir_b200_sync", "ipir_b200_enable_stage_timing",
    "ipir_b200_stage_times", "ipir_b200_export_precomp", "ipir_b200_export_db", "ipir_b200_ntt",
    "ipir_b200_decomp", "ipir_b200_shake256", "ipir_b200_expand_seed", "ipir_b200_fill_db",
    "ipir_b200_matvec", "ipir_b200_matvec_noalloc", "ipir_b200_autotune", "ipir_b200_get_schedule",
    "ipir_b200_launch_count", "ipir_serve_create", "ipir_serve_submit", "ipir_serve_poll", "ipir_serve_wait",
    "ipir_serve_stats", "ipir_serve_db_info", "ipir_serve_trace", "ipir_serve_destroy", "ipir_b200_matvec_ex",
    "ipir_b200_fill_db_device", "ipir_b200_set_schedule", "ipir_b200_wire_sizes", "ipir_b200_answer_wire",
    "ipir_serve_replace_db", "ipir_b200_save_server", "ipir_b200_load_server",
    "ipir_b200_kernel_binary_version", "ipir_b200_shard_create", "ipir_b200_shard_export_a",
    "ipir_b200_shard_pack", "ipir_b200_shard_destroy", "ipir_b200_horner_create", "ipir_b200_horner_answer",
    "ipir_b200_horner_destroy", "ipir_b200_synth_queries", "ipir_b200_horner_eval", "ipir_b200_shard_answer",
]


class InspireError(RuntimeError):
    pass


def last_error():
    return _L.ipir_b200_last_error().decode()


def _ptr(a, t):
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data_as(t)


def library_handle():
    return _L


def setup(n_entries, entry_bytes, db_rows=0):
    """Geometry of the reference's setup() (src/params.cpp:23-68).  Raises
    ValueError where the reference throws std::invalid_argument."""
    p = IpirParams()
    rc = _L.ipir_b200_setup(n_entries, entry_bytes, db_rows, C.byref(p))
    if rc:
        raise ValueError(last_error())
    return p.as_dict()


def query_u64s(params):
    return 2 * params["db_rows"] + 6 * D_EFF * 2 * RING_N


def response_u64s(params):
    return params["num_cts"] * 4 * RING_N


def query_view_from_flat(params, flat):
    """View into a flat query (reference ipir_query_view_from_flat,
    src/capi_client.cpp:81-93).  ``flat`` must stay alive while the view is used."""
    flat = np.ascontiguousarray(flat, dtype=np.uint64)
    if flat.size != query_u64s(params):
        raise ValueError(f"flat query has {flat.size} u64, expected {query_u64s(params)}")
    R = params["db_rows"]
    blk = D_EFF * 2 * RING_N
    base = flat.ctypes.data
    v = IpirQueryView()
    v.lwe_b_limb0 = C.cast(base, u64p)
    v.lwe_b_limb1 = C.cast(base + 8 * R, u64p)
    v.ksk5_b = C.cast(base + 8 * (2 * R), u64p)
    v.kskneg1_b = C.cast(base + 8 * (2 * R + blk), u64p)
    v.rgsw = C.cast(base + 8 * (2 * R + 2 * blk), u64p)
    return v


class Server:
    """One database generation on the current CUDA device (reference
    ipir_server_create / GpuServerCtx)."""

    def __init__(self, n_entries, entry_bytes, db, db_rows=0, max_batch=16, crs_seed=None):
        db = np.ascontiguousarray(db, dtype=np.uint16)
        p = IpirParams()
        seed = None
        if crs_seed is not None:
            if len(crs_seed) != 64:
                raise ValueError("crs_seed must be 64 bytes")
            seed = np.frombuffer(bytes(crs_seed), np.uint8).copy()
        h = _L.ipir_server_create(n_entries, entry_bytes, db_rows, max_batch, _ptr(db, u16p),
                                  _ptr(seed, u8p) if seed is not None else None, C.byref(p))
        if not h:
            raise InspireError(f"ipir_server_create failed: {last_error()}")
        self._h = h
        self.params = p.as_dict()
        self.max_batch = max_batch

    @classmethod
    def load(cls, path, max_batch=16):
        """A handle restored from a checkpoint written by save() (no raw DB,
        no preprocessing); raises InspireError for a missing, truncated,
        foreign or corrupted file."""
        p = IpirParams()
        h = _L.ipir_b200_load_server(os.fsencode(path), max_batch, C.byref(p))
        if not h:
            raise InspireError(f"ipir_b200_load_server failed: {last_error()}")
        self = cls.__new__(cls)
        self._h = h
        self.params = p.as_dict()
        self.max_batch = max_batch
        return self

    def save(self, path):
        """Write this handle's resident state (encoded DB, precomputed
        tensors, public parameters) to `path`."""
        self._check()
        rc = _L.ipir_b200_save_server(self._h, os.fsencode(path))
        if rc:
            raise InspireError(f"ipir_b200_save_server rc={rc}: {last_error()}")

    def _check(self):
        if not self._h:
            raise InspireError("server destroyed")

    def caps(self):
        self._check()
        c = IpirCaps()
        _L.ipir_server_caps(self._h, C.byref(c))
        return {f: getattr(c, f) for f, _ in c._fields_}

    def _views(self, queries):
        flats = [np.ascontiguousarray(q, dtype=np.uint64) for q in queries]
        arr = (IpirQueryView * max(1, len(flats)))()
        for i, f in enumerate(flats):
            arr[i] = query_view_from_flat(self.params, f)
        return arr, flats

    def answer_batch(self, queries, out=None):
        """queries: list of flat u64 queries -> (count, num_cts*4*N) u64 responses."""
        self._check()
        views, keep = self._views(queries)
        n = len(keep)
        if out is None:
            out = np.zeros((n, response_u64s(self.params)), np.uint64)
        rc = _L.ipir_answer_batch(self._h, views, n, _ptr(out, u64p))
        if rc:
            raise InspireError(f"ipir_answer_batch rc={rc}: {last_error()}")
        return out

    def answer(self, query):
        return self.answer_batch([query])[0]

    def answer_batch_rc(self, views, count, out):
        """Raw C call returning the reference's code (tests of the error contract)."""
        return _L.ipir_answer_batch(self._h, views, count, _ptr(out, u64p) if out is not None else None)

    # device-resident pipeline --------------------------------------------
    def set_stream(self, stream_handle):
        self._check()
        _L.ipir_b200_set_stream(self._h, C.c_void_p(stream_handle or 0))

    def stage(self, queries):
        self._check()
        views, keep = self._views(queries)
        self._staged_keep = keep
        rc = _L.ipir_b200_stage_queries(self._h, views, len(keep))
        if rc:
            raise InspireError(f"stage rc={rc}: {last_error()}")

    def stage_views(self, views, count):
        rc = _L.ipir_b200_stage_queries(self._h, views, count)
        if rc:
            raise InspireError(f"stage rc={rc}: {last_error()}")

    def run(self, count):
        self._check()
        rc = _L.ipir_b200_run(self._h, count)
        if rc:
            raise InspireError(f"run rc={rc}: {last_error()}")

    def fetch(self, count, out=None):
        self._check()
        if out is None:
            out = np.zeros((count, response_u64s(self.params)), np.uint64)
        rc = _L.ipir_b200_fetch_responses(self._h, count, _ptr(out, u64p))
        if rc:
            raise InspireError(f"fetch rc={rc}: {last_error()}")
        return out

    def sync(self):
        self._check()
        if _L.ipir_b200_sync(self._h):
            raise InspireError(last_error())

    def enable_stage_timing(self, on=True):
        _L.ipir_b200_enable_stage_timing(self._h, 1 if on else 0)

    def stage_times(self):
        a = (C.c_float * 5)()
        _L.ipir_b200_stage_times(self._h, a, 5)
        return dict(zip(["qprep", "matvec", "collapse", "finalize", "horner"], list(a)))

    def export_precomp(self, group):
        self._check()
        a = np.zeros(2 * RING_N, np.uint32)
        dp = np.zeros(2 * NSTEPS * D_EFF * RING_N, np.uint32)
        dm = np.zeros_like(dp)
        df = np.zeros(2 * D_EFF * RING_N, np.uint32)
        rc = _L.ipir_b200_export_precomp(self._h, group, _ptr(a, u32p), _ptr(dp, u32p),
                                         _ptr(dm, u32p), _ptr(df, u32p))
        if rc:
            raise InspireError(f"export_precomp rc={rc}: {last_error()}")
        return a, dp, dm, df

    def export_db(self, row0, nrows):
        self._check()
        out = np.zeros(nrows * self.params["db_cols"], np.uint16)
        rc = _L.ipir_b200_export_db(self._h, row0, nrows, _ptr(out, u16p))
        if rc:
            raise InspireError(f"export_db rc={rc}: {last_error()}")
        return out

    # wire formats ------------------------------------------------------
    def wire_sizes(self):
        """(packed query, packed response, compressed response) bytes per query."""
        p = IpirParams()
        for k, v in self.params.items():
            if k == "seed":
                p.seed[:] = list(v)
            else:
                setattr(p, k, v)
        a, b_, c = C.c_size_t(), C.c_size_t(), C.c_size_t()
        _L.ipir_b200_wire_sizes(C.byref(p), C.byref(a), C.byref(b_), C.byref(c))
        return a.value, b_.value, c.value

    def answer_wire(self, packed, count, resp_format=RESP_COMPRESSED, out=None):
        """Answer `count` packed queries (uint8, count x packed-query bytes);
        returns the responses in resp_format (u64 rows for RESP_FLAT, bytes otherwise)."""
        self._check()
        qb, rb, cb = self.wire_sizes()
        packed = np.ascontiguousarray(packed, dtype=np.uint8).reshape(-1)
        if packed.size != count * qb:
            raise ValueError(f"packed queries: {packed.size} bytes, expected {count * qb}")
        if out is None:
            out = (np.zeros((count, response_u64s(self.params)), np.uint64) if resp_format == RESP_FLAT else
                   np.zeros((count, rb if resp_format == RESP_PACKED else cb), np.uint8))
        rc = _L.ipir_b200_answer_wire(self._h, packed.ctypes.data, count, resp_format, out.ctypes.data)
        if rc:
            raise InspireError(f"answer_wire rc={rc}: {last_error()}")
        return out

    # schedules ---------------------------------------------------------
    def autotune(self):
        """Time the candidate kernel schedules per batch size; later calls use the fastest."""
        self._check()
        if _L.ipir_b200_autotune(self._h):
            raise InspireError(f"autotune: {last_error()}")

    def schedule(self, count):
        self._check()
        s = IpirSchedule()
        rc = _L.ipir_b200_get_schedule(self._h, count, C.byref(s))
        if rc:
            raise InspireError(f"get_schedule rc={rc}")
        return s.as_dict()

    def set_schedule(self, count, matvec_tc=1, tp_pass=None, horner_cluster=1, tp_sms=0, slice=32, hchunks=0):
        """Pin the kernel schedule for batches of `count` queries (tp_sms > 0:
        tensor pass on that many SMs beside the mat-vec; slice 32: batches of
        more than 32 run as consecutive 32-query pipelines, 0: one pipeline;
        hchunks 2..16: the Horner chain trails the DB pass in at most that
        many group chunks)."""
        self._check()
        s = IpirSchedule(matvec_tc, tp_pass if tp_pass is not None else self.schedule(count)["tp_pass"],
                         horner_cluster, tp_sms, slice, hchunks)
        rc = _L.ipir_b200_set_schedule(self._h, count, C.byref(s))
        if rc:
            raise InspireError(f"set_schedule rc={rc}: {last_error()}")

    def launch_count(self):
        """Kernels launched by this handle's answer pipeline so far."""
        v = C.c_ulonglong()
        _L.ipir_b200_launch_count(self._h, C.byref(v))
        return v.value

    def close(self):
        if self._h:
            _L.ipir_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ serving loop
SERVE_DONE, SERVE_PENDING, SERVE_UNKNOWN, SERVE_FAILED, SERVE_TIMEOUT, SERVE_FULL = 0, 1, 2, 4, 5, 6


class ServeLoop:
    """Continuous-batching serving loop over resident databases (the
    ipir_serve_* entry points): submit() returns a ticket at once; poll() /
    wait() collect the response and its submit-to-response latency.
    scan_segments > 1: cyclic scan (requests join the running rotation of
    DB-pass segments) for the databases whose groups split that way; < 0:
    per database, cyclic scan when its plain answer takes 2 ms or more."""

    def __init__(self, servers, max_batch=0, lanes_per_db=0, queue_slots=0, hbm_budget_bytes=0,
                 graphs=True, autotune=True, overlap_db_passes=False, scan_segments=0):
        self.servers = list(servers)
        hs = (C.c_void_p * len(self.servers))(*[s._h for s in self.servers])
        cfg = IpirServeConfig(max_batch, lanes_per_db, queue_slots, hbm_budget_bytes,
                              0 if graphs else 1, 0 if autotune else 1, 1 if overlap_db_passes else 0,
                              scan_segments)
        h = _L.ipir_serve_create(hs, len(self.servers), C.byref(cfg))
        if not h:
            raise InspireError(f"ipir_serve_create failed: {last_error()}")
        self._h = h

    def submit_view(self, db, view):
        """Returns (rc, ticket); rc 6 means every request slot is in use."""
        t = C.c_uint64()
        rc = _L.ipir_serve_submit(self._h, db, C.byref(view), C.byref(t))
        return rc, t.value

    def submit(self, db, flat_query):
        v = query_view_from_flat(self.servers[db].params, flat_query)
        rc, t = self.submit_view(db, v)
        if rc:
            raise InspireError(f"submit rc={rc}: {last_error() if rc == 4 else ''}")
        return t

    def poll(self, ticket, out=None):
        """(rc, latency_ms); rc SERVE_DONE writes the response into out (if given)."""
        lat = C.c_double()
        rc = _L.ipir_serve_poll(self._h, ticket, _ptr(out, u64p) if out is not None else None, C.byref(lat), None)
        return rc, lat.value

    def wait(self, ticket, out=None, timeout=60.0, with_queue=False):
        """Latency in ms (submit to response); with_queue: (latency, submit-to-launch)."""
        lat, qms = C.c_double(), C.c_double()
        rc = _L.ipir_serve_wait(self._h, ticket, timeout, _ptr(out, u64p) if out is not None else None,
                                C.byref(lat), C.byref(qms))
        if rc:
            raise InspireError(f"wait rc={rc}: {last_error() if rc == 4 else ''}")
        return (lat.value, qms.value) if with_queue else lat.value

    def stats(self):
        c = IpirServeCounters()
        _L.ipir_serve_stats(self._h, C.byref(c))
        return {f: getattr(c, f) for f, _ in c._fields_}

    def replace_db(self, db, server):
        """Switch database `db` to the next generation `server` (same geometry)."""
        rc = _L.ipir_serve_replace_db(self._h, db, server._h)
        if rc:
            raise InspireError(f"replace_db rc={rc}: {last_error()}")
        self.servers[db] = server

    def trace(self, max_records=4096):
        """The most recent lane batches, oldest first (dicts of ipir_serve_batch_record)."""
        buf = (IpirServeBatchRecord * max_records)()
        n = _L.ipir_serve_trace(self._h, buf, max_records)
        return [{f: getattr(buf[i], f) for f, _ in IpirServeBatchRecord._fields_} for i in range(n)]

    def db_info(self, db):
        lanes, mb = C.c_size_t(), C.c_size_t()
        tab = (IpirSchedule * 65)()
        _L.ipir_serve_db_info(self._h, db, C.byref(lanes), C.byref(mb), tab, 65)
        return {"lanes": lanes.value, "max_batch": mb.value,
                "schedule": {c: tab[c].as_dict() for c in range(1, min(64, mb.value) + 1)}}

    def close(self):
        if self._h:
            _L.ipir_serve_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ primitives
def ntt(polys, limb_run=1, inverse=False):
    """GPU forward/inverse NTT of (n, 2048) u32 residues; poly i is mod
    q_((i // limb_run) & 1)."""
    a = np.ascontiguousarray(polys, dtype=np.uint32).copy()
    n = a.size // RING_N
    rc = _L.ipir_b200_ntt(_ptr(a, u32p), n, limb_run, 1 if inverse else 0)
    if rc:
        raise InspireError(f"ipir_b200_ntt rc={rc}: {last_error()}")
    return a


def decomp(polys):
    """GPU gadget decomposition: (n, 2, 2048) coefficient form -> (n, 2, 2, 2048)
    [digit][limb]."""
    a = np.ascontiguousarray(polys, dtype=np.uint32)
    n = a.size // (2 * RING_N)
    out = np.zeros(n * D_EFF * 2 * RING_N, np.uint32)
    rc = _L.ipir_b200_decomp(_ptr(a, u32p), _ptr(out, u32p), n)
    if rc:
        raise InspireError(f"ipir_b200_decomp rc={rc}: {last_error()}")
    return out


def shake256(data, outlen):
    src = np.frombuffer(bytes(data), np.uint8).copy() if len(data) else np.zeros(1, np.uint8)
    out = np.zeros(max(outlen, 1), np.uint8)
    _L.ipir_b200_shake256(_ptr(src, u8p), len(data), _ptr(out, u8p), outlen)
    return out[:outlen].tobytes()


def expand_seed(seed, domain, index):
    s = np.frombuffer(bytes(seed), np.uint8).copy()
    out = np.zeros(2 * RING_N, np.uint32)
    rc = _L.ipir_b200_expand_seed(_ptr(s, u8p), domain.encode(), index, _ptr(out, u32p))
    if rc:
        raise InspireError(last_error())
    return out


def fill_db(count, seed, out=None):
    """Synthetic DB: splitmix64(seed ^ k) mod 65535 (host, all threads)."""
    if out is None:
        out = np.empty(count, np.uint16)
    _L.ipir_b200_fill_db(_ptr(out, u16p), count, seed)
    return out


def matvec(db_ptr, rows, cols, queries_ptr, count, out_ptr, stream=0, sync=True):
    """Exact tensor-core mat-vec on device pointers (ints):
    out[q][limb][c] = sum_i db[i][c] * queries[q][limb][i] mod q_limb."""
    rc = _L.ipir_b200_matvec(C.c_void_p(db_ptr), rows, cols, C.c_void_p(queries_ptr), count,
                             C.c_void_p(out_ptr), C.c_void_p(stream or 0), 1 if sync else 0)
    if rc:
        raise InspireError(f"ipir_b200_matvec rc={rc}: {last_error()}")


def matvec_ex(db_ptr, rows, cols, queries_ptr, count, out_ptr, path=0, queries_per_pass=0, kchunk_rows=0,
              stream=0, sync=True):
    """ipir_b200_matvec_ex: the mat-vec with an explicit schedule (path 0 =
    tensor cores, 1 = CUDA cores); device pointers as in matvec()."""
    o = IpirMatvecOpts(path, queries_per_pass, kchunk_rows)
    rc = _L.ipir_b200_matvec_ex(C.c_void_p(db_ptr), rows, cols, C.c_void_p(queries_ptr), count, C.c_void_p(out_ptr),
                                C.c_void_p(stream or 0), 1 if sync else 0, C.byref(o))
    if rc:
        raise InspireError(f"matvec_ex rc={rc}: {last_error()}")


def fill_db_device(ptr, count, seed, stream=0):
    """Device-side fill_db (same values) into device memory at ptr."""
    rc = _L.ipir_b200_fill_db_device(C.c_void_p(ptr), count, seed, C.c_void_p(stream or 0))
    if rc:
        raise InspireError(f"fill_db_device rc={rc}: {last_error()}")


def synth_queries_device(db_rows, seed, first_id, count, out_ptr, stream=0):
    """Synthetic flat queries (uniform residues per limb) for ids first_id ..
    first_id + count - 1, written by a kernel into device memory at out_ptr
    (enqueued on `stream`)."""
    rc = _L.ipir_b200_synth_queries(db_rows, seed, first_id, count, C.c_void_p(out_ptr), C.c_void_p(stream or 0))
    if rc:
        raise InspireError(f"synth_queries rc={rc}: {last_error()}")


def synth_queries_host(db_rows, seed, first_id, count):
    """The same values computed on the host (numpy), for checks."""
    qn = 2 * db_rows + 6 * D_EFF * 2 * RING_N
    k = np.arange(qn, dtype=np.uint64)
    limb = np.where(k < db_rows, 0, np.where(k < 2 * db_rows, 1, ((k - 2 * db_rows) // RING_N) & 1))
    q = np.where(limb == 1, np.uint64(Q1), np.uint64(Q0)).astype(np.uint64)
    out = np.empty((count, qn), np.uint64)
    with np.errstate(over="ignore"):
        for j in range(count):
            h = _splitmix64(np.uint64(seed) ^ (np.uint64(first_id + j) * np.uint64(0xD1B54A32D192ED03)))
            out[j] = _splitmix64(h ^ k) % q
    return out


def _splitmix64(x):
    with np.errstate(over="ignore"):
        x = np.asarray(x, np.uint64) + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return x ^ (x >> np.uint64(31))


def horner_eval(rgsw, cts, L, variant=1):
    """HornerEval on host arrays through the server's Horner kernels
    (variant 0: one CTA, 1: 4-CTA cluster, 2: 8-CTA cluster); returns 4 N u64."""
    rgsw = np.ascontiguousarray(rgsw, np.uint64)
    cts = np.ascontiguousarray(cts, np.uint64)
    if rgsw.size != 4 * D_EFF * 2 * RING_N or cts.size != L * 4 * RING_N:
        raise ValueError("rgsw must hold 4 * D_EFF * 2 * N u64 and cts L * 4 * N u64")
    out = np.zeros(4 * RING_N, np.uint64)
    rc = _L.ipir_b200_horner_eval(_ptr(rgsw, u64p), _ptr(cts, u64p), L, _ptr(out, u64p), variant)
    if rc:
        raise InspireError(f"horner_eval rc={rc}: {last_error()}")
    return out


def kernel_binary_version():
    """cudaFuncAttributes.binaryVersion of the library's kernels as loaded
    (100 for sm_100a)."""
    v = C.c_int(0)
    rc = _L.ipir_b200_kernel_binary_version(C.byref(v))
    if rc:
        raise InspireError(f"ipir_b200_kernel_binary_version rc={rc}: {last_error()}")
    return v.value


def matvec_noalloc_rc(db_ptr, rows, cols, queries_ptr, count, out_ptr, stream=0):
    """ipir_b200_matvec_noalloc on device pointers; returns the C return code.
    Allocates nothing: its scratch is a fixed array in the library (rows <=
    32768, count <= 8); the first call on a device sets it up."""
    return _L.ipir_b200_matvec_noalloc(C.c_void_p(db_ptr), rows, cols, C.c_void_p(queries_ptr), count,
                                       C.c_void_p(out_ptr), C.c_void_p(stream or 0))


# ------------------------------------------------------------------ group shards
def chunk_ranges(n_packed, d_act, world):
    """Group ranges of whole Horner chunks (response ciphertexts) over
    `world` GPUs, contiguous and as even as possible, for databases of at
    least `world` ciphertexts: every rank answers its ciphertexts, with no
    exchange before Horner."""
    n_cts = -(-n_packed // d_act)
    if world < 1 or world > n_cts:
        raise ValueError(f"cannot split {n_cts} ciphertexts over {world} shards")
    base, extra = divmod(n_cts, world)
    out, c = [], 0
    for r in range(world):
        c1 = c + base + (1 if r < extra else 0)
        out.append((c * d_act, min(n_packed, c1 * d_act)))
        c = c1
    return out


def group_ranges(n_packed, world):
    """Contiguous group ranges [lo, hi) of a database split over `world`
    GPUs, as equal as possible (the first n_packed % world get one more)."""
    if world < 1 or world > n_packed:
        raise ValueError(f"cannot split {n_packed} groups over {world} shards")
    base, extra = divmod(n_packed, world)
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


class Shard:
    """Groups [lo, hi) of one database on the current CUDA device
    (ipir_b200_shard_create): pack() gives the b parts of those groups'
    packed ciphertexts for a batch, in device memory."""

    def __init__(self, n_entries, entry_bytes, db, group_lo, group_hi, crs_seed, db_rows=0, max_batch=16):
        db = np.ascontiguousarray(db, dtype=np.uint16)
        if len(crs_seed) != 64:
            raise ValueError("crs_seed must be 64 bytes")
        seed = np.frombuffer(bytes(crs_seed), np.uint8).copy()
        p = IpirParams()
        h = _L.ipir_b200_shard_create(n_entries, entry_bytes, db_rows, max_batch, _ptr(db, u16p), _ptr(seed, u8p),
                                      group_lo, group_hi, C.byref(p))
        if not h:
            raise InspireError(f"ipir_b200_shard_create failed: {last_error()}")
        self._h = h
        self.params = p.as_dict()
        self.lo, self.hi = group_lo, group_hi
        self.max_batch = max_batch

    @property
    def groups(self):
        return self.hi - self.lo

    def packed_u32s(self, count):
        return count * self.groups * 2 * RING_N

    def export_a(self):
        out = np.zeros(self.groups * 2 * RING_N, np.uint32)
        rc = _L.ipir_b200_shard_export_a(self._h, _ptr(out, u32p))
        if rc:
            raise InspireError(f"shard_export_a rc={rc}: {last_error()}")
        return out

    def pack(self, queries, out_ptr):
        """queries: flat u64 queries; out_ptr: device pointer (int) to
        count * groups * 2 * N u32 ([query][group][limb][N])."""
        arr = (IpirQueryView * max(1, len(queries)))()
        keep = [np.ascontiguousarray(q, np.uint64) for q in queries]
        for i, f in enumerate(keep):
            arr[i] = query_view_from_flat(self.params, f)
        rc = _L.ipir_b200_shard_pack(self._h, arr, len(keep), C.c_void_p(out_ptr))
        if rc:
            raise InspireError(f"shard_pack rc={rc}: {last_error()}")

    def cts(self):
        """Response ciphertexts this shard answers itself (0 if its range does
        not cover whole Horner chunks)."""
        d_act = min(self.params["interp_d"], self.params["n_packed"])
        whole = self.lo % d_act == 0 and (self.hi % d_act == 0 or self.hi == self.params["n_packed"])
        return -(-self.groups // d_act) if whole else 0

    def answer(self, queries, out=None):
        """Its own ciphertexts of each query's response (whole-chunk shards):
        (count, cts * 4 N) u64."""
        keep = [np.ascontiguousarray(q, np.uint64) for q in queries]
        arr = (IpirQueryView * max(1, len(keep)))()
        for i, f in enumerate(keep):
            arr[i] = query_view_from_flat(self.params, f)
        if out is None:
            out = np.zeros((len(keep), self.cts() * 4 * RING_N), np.uint64)
        rc = _L.ipir_b200_shard_answer(self._h, arr, len(keep), _ptr(out, u64p))
        if rc:
            raise InspireError(f"shard_answer rc={rc}: {last_error()}")
        return out

    def close(self):
        if self._h:
            _L.ipir_b200_shard_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HornerOwner:
    """The Horner chains of a sharded database (ipir_b200_horner_create) on
    the current CUDA device, from the gathered b parts of every group."""

    def __init__(self, params, a_all, max_batch=16):
        p = IpirParams()
        for f, _ in IpirParams._fields_:
            if f == "seed":
                p.seed[:] = list(params["seed"])
            else:
                setattr(p, f, params[f])
        a_all = np.ascontiguousarray(a_all, np.uint32)
        if a_all.size != params["n_packed"] * 2 * RING_N:
            raise ValueError("a_all must hold n_packed * 2 * N u32")
        h = _L.ipir_b200_horner_create(C.byref(p), _ptr(a_all, u32p), max_batch)
        if not h:
            raise InspireError(f"ipir_b200_horner_create failed: {last_error()}")
        self._h = h
        self.params = dict(params)
        self.max_batch = max_batch

    def answer(self, packed_ptr, queries, stream=0, out=None):
        """packed_ptr: device pointer to count * n_packed * 2 * N u32; returns
        (count, num_cts * 4 * N) u64 responses."""
        keep = [np.ascontiguousarray(q, np.uint64) for q in queries]
        arr = (IpirQueryView * max(1, len(keep)))()
        for i, f in enumerate(keep):
            arr[i] = query_view_from_flat(self.params, f)
        if out is None:
            out = np.zeros((len(keep), response_u64s(self.params)), np.uint64)
        rc = _L.ipir_b200_horner_answer(self._h, C.c_void_p(packed_ptr), arr, len(keep), _ptr(out, u64p),
                                        C.c_void_p(stream or 0))
        if rc:
            raise InspireError(f"horner_answer rc={rc}: {last_error()}")
        return out

    def close(self):
        if self._h:
            _L.ipir_b200_horner_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
