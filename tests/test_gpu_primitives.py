"""GPU primitives against the reference's own CPU code, bit-exact (the
reference's tests/test_gpu_ntt.cu, tests/test_gpu_decomp.cu)."""
import numpy as np
import pytest

from oracle_lib import N, QS

pytestmark = pytest.mark.gpu


def _rand_polys(rng, n, limb_run):
    a = np.zeros((n, N), np.uint32)
    for i in range(n):
        a[i] = rng.integers(0, QS[(i // limb_run) & 1], N, dtype=np.uint32)
    return a


@pytest.mark.parametrize("limb_run", [1, 2, 64])
def test_ntt_forward_matches_reference(ref, limb_run):
    import inspire_b200 as ib
    rng = np.random.default_rng(42)
    a = _rand_polys(rng, 256, limb_run)
    got = ib.ntt(a, limb_run=limb_run).reshape(256, N)
    for i in range(256):
        exp = ref.ntt_forward(a[i].astype(np.uint64), (i // limb_run) & 1)
        assert (got[i].astype(np.uint64) == exp).all(), i


def test_ntt_inverse_and_roundtrip(ref):
    import inspire_b200 as ib
    rng = np.random.default_rng(7)
    a = _rand_polys(rng, 64, 1)
    inv = ib.ntt(a, limb_run=1, inverse=True).reshape(64, N)
    for i in range(64):
        assert (inv[i].astype(np.uint64) == ref.ntt_inverse(a[i].astype(np.uint64), i & 1)).all(), i
    back = ib.ntt(ib.ntt(a, 1), 1, inverse=True).reshape(64, N)
    assert (back == a).all()


def test_ntt_edge_values(ref):
    import inspire_b200 as ib
    a = np.zeros((4, N), np.uint32)
    a[0] = QS[0] - 1
    a[1] = QS[1] - 1
    a[2, 0] = 1
    a[3, N - 1] = QS[1] - 1
    got = ib.ntt(a, 1).reshape(4, N)
    for i in range(4):
        assert (got[i].astype(np.uint64) == ref.ntt_forward(a[i].astype(np.uint64), i & 1)).all()


def test_decomp_matches_reference(ref):
    import inspire_b200 as ib
    rng = np.random.default_rng(42)
    n = 16
    f = np.zeros((n, 2, N), np.uint32)
    f[:, 0] = rng.integers(0, QS[0], (n, N), dtype=np.uint32)
    f[:, 1] = rng.integers(0, QS[1], (n, N), dtype=np.uint32)
    f[0, :, :4] = 0                              # zero
    f[1, 0, :4], f[1, 1, :4] = QS[0] - 1, QS[1] - 1  # -1
    got = ib.decomp(f).reshape(n, 2 * 2 * N)
    for i in range(n):
        assert (got[i].astype(np.uint64) == ref.decomp(f[i].reshape(-1).astype(np.uint64))).all(), i


def test_kernels_loaded_as_sm100():
    """The CUDA runtime loaded the library's sm_100a cubin (binaryVersion 100)."""
    import inspire_b200 as ib
    assert ib.kernel_binary_version() == 100


def test_synth_queries_kernel_matches_host_formula():
    """The load generator's kernel writes what its host restatement gives,
    residues below each word's limb modulus, distinct per query id."""
    import torch
    import inspire_b200 as ib
    rows, n, first = 2048, 3, 1_000_003
    qn = ib.query_u64s({"db_rows": rows})
    buf = torch.zeros(n * qn, dtype=torch.int64, device="cuda")
    ib.synth_queries_device(rows, 77, first, n, buf.data_ptr())
    torch.cuda.synchronize()
    got = buf.cpu().numpy().view(np.uint64).reshape(n, qn)
    want = ib.synth_queries_host(rows, 77, first, n)
    assert (got == want).all()
    assert (got[:, :rows] < QS[0]).all() and (got[:, rows:2 * rows] < QS[1]).all()
    assert not (got[0] == got[1]).all()
