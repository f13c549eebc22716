"""Host-side checks of the product library without a GPU: it loads, exports
every symbol include/*.h declares, and its host logic (setup geometry,
SHAKE-256, expand_seed, synthetic DB) matches the reference / standard."""
import hashlib
import os
import re

import numpy as np
import pytest

from oracle_lib import REPO, crs_seed_from


def header_symbols():
    txt = open(os.path.join(REPO, "include", "inspire_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ipir_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    import inspire_b200 as ib
    L = ib.library_handle()
    syms = header_symbols()
    assert "ipir_server_create" in syms and "ipir_answer_batch" in syms
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(ib.EXPORTED) == syms


def test_library_is_built_for_sm100a_only():
    """Every device-code compile and the link name the one target
    (-gencode arch=compute_100a,code=sm_100a) and no other; the GPU test
    test_gpu_primitives.py::test_kernels_loaded_as_sm100 reads the target
    back from the loaded module."""
    mk = open(os.path.join(REPO, "inspire-gpu_b200", "Makefile")).read()
    arch_lines = [l for l in mk.splitlines() if "arch=" in l or "-arch" in l or "code=" in l]
    assert arch_lines and all("arch=compute_100a,code=sm_100a" in l for l in arch_lines), arch_lines
    assert set(re.findall(r"(?:sm|compute)_(\d+a?)", mk)) == {"100a"}


def test_reference_client_symbols_not_defined():
    import inspire_b200 as ib
    L = ib.library_handle()
    for s in ("ipir_query_build", "ipir_extract", "ipir_query_pack"):
        assert not hasattr(L, s), s


@pytest.mark.parametrize("args", [(65536, 30, 0), (256, 120, 2048), (262144, 120, 2048),
                                  (1 << 25, 30, 0), (1 << 29, 30, 0), (1 << 22, 960, 0),
                                  (1 << 31, 30, 0), (1000, 30, 0), (5, 2, 2048)])
def test_setup_matches_reference(ref, args):
    import inspire_b200 as ib
    p = ib.setup(*args)
    assert [p[k] for k in ("n_entries", "entry_bytes", "db_rows", "db_cols", "n_packed",
                           "interp_d", "num_cts")] == ref.setup(*args)


@pytest.mark.parametrize("args", [(1 << 25, 32, 0), (1 << 22, 1024, 0), (196608, 120, 2048), (25165824, 120, 2048)])
def test_setup_rejects_what_reference_rejects(ref, args):
    import inspire_b200 as ib
    with pytest.raises(ValueError):
        ref.setup(*args)
    with pytest.raises(ValueError):
        ib.setup(*args)


def test_shake256_matches_hashlib():
    import inspire_b200 as ib
    for n in (0, 1, 135, 136, 137, 272, 500):
        d = bytes((i * 7 + 3) & 0xFF for i in range(n))
        for ol in (1, 32, 136, 137, 4096):
            assert ib.shake256(d, ol) == hashlib.shake_256(d).digest(ol), (n, ol)


def test_expand_seed_matches_reference(ref):
    import inspire_b200 as ib
    seed = crs_seed_from(9)
    for dom, idx in (("rlwe", 0), ("rlwe", 31), ("ksk", 502), ("ksk", 409501)):
        assert (ib.expand_seed(seed, dom, idx).astype(np.uint64) == ref.expand_seed(seed, dom, idx)).all()


def test_fill_db_matches_oracle(oracle):
    import inspire_b200 as ib
    assert (ib.fill_db(100003, 11) == oracle.fill_db(100003, 11)).all()


def test_server_create_rejects_bad_args_without_gpu_work():
    import inspire_b200 as ib
    with pytest.raises(ib.InspireError):
        ib.Server(1 << 25, 32, np.zeros(16, np.uint16))   # geometry rejected before any device call


def test_serve_entry_points_reject_null_without_gpu_work():
    import ctypes as C
    import inspire_b200 as ib
    L = ib.library_handle()
    assert not L.ipir_serve_create(None, 0, None)
    assert "no databases" in ib.last_error()
    t = C.c_uint64()
    assert L.ipir_serve_submit(None, 0, None, C.byref(t)) == 1
    assert L.ipir_serve_poll(None, 1, None, None, None) == 1
    assert L.ipir_serve_wait(None, 1, 0.0, None, None, None) == 1
    assert L.ipir_serve_stats(None, None) == 1
    assert L.ipir_serve_db_info(None, 0, None, None, None, 0) == 1
    L.ipir_serve_destroy(None)
    s = ib.IpirSchedule()
    assert L.ipir_b200_get_schedule(None, 1, C.byref(s)) == 1
    assert L.ipir_b200_autotune(None) == 1
    v = C.c_ulonglong()
    assert L.ipir_b200_launch_count(None, C.byref(v)) == 1


@pytest.mark.parametrize("args", [(256, 120, 2048), (262144, 120, 2048), (65536, 30, 0), (1 << 29, 30, 0)])
def test_wire_sizes_match_reference_client(ref, args):
    import ctypes as C
    import inspire_b200 as ib
    from oracle_lib import crs_seed_from, ref_params
    g = ref.setup(*args)
    rp = ref_params(g, args[:2], crs_seed_from(1))
    p = ib.IpirParams()
    assert ib.library_handle().ipir_b200_setup(args[0], args[1], args[2], C.byref(p)) == 0
    a, b, c = C.c_size_t(), C.c_size_t(), C.c_size_t()
    assert ib.library_handle().ipir_b200_wire_sizes(C.byref(p), C.byref(a), C.byref(b), C.byref(c)) == 0
    L = ref.L
    assert (a.value, b.value, c.value) == (L.ipir_query_packed_bytes(C.byref(rp)),
                                           L.ipir_response_packed_bytes(C.byref(rp)),
                                           L.ipir_response_compressed_bytes(C.byref(rp)))


def test_reference_cpp_consumer_links_this_projects_library():
    """The reference-typed C++ API: the consumer built against it resolves
    the reference's server functions from libinspire_b200_refapi.so (over
    libinspire_b200.so), not from the reference's GPU library."""
    import subprocess
    exe = os.path.join(REPO, "oracle", "_ref", "ref_consumer_b200")
    if not os.path.exists(exe):
        pytest.skip("consumer not built (needs the reference's headers)")
    out = subprocess.run(["ldd", exe], capture_output=True, text=True).stdout
    assert "libinspire_b200_refapi.so" in out and "libinspire_b200.so" in out and "not found" not in out
    assert "libinspire_ref_gpu" not in out


def test_synth_queries_host_formula_ranges():
    import inspire_b200 as ib
    from oracle_lib import Q0, Q1
    rows = 4096
    q = ib.synth_queries_host(rows, 5, 0, 2)
    blocks = q[:, 2 * rows:].reshape(2, -1, 2048)
    assert (q[:, :rows] < Q0).all() and (q[:, rows:2 * rows] < Q1).all()
    assert (blocks[:, 0::2] < Q0).all() and (blocks[:, 1::2] < Q1).all()
    assert (q[:, rows:2 * rows] >= Q0).any()          # limb 1 uses its own modulus
    assert (ib.synth_queries_host(rows, 5, 1, 1)[0] == q[1]).all()   # a query regenerates from its id
