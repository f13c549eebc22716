"""The server's ExtProd / Horner kernels alone against the reference's own
CPU ext_prod and horner_eval (src/crypto.cpp:219-279), bit-exact, as the
reference's tests/test_gpu_extprod.cu and tests/test_gpu_horner.cu pin its
GPU versions: every kernel variant (one CTA, 4-CTA and 8-CTA clusters),
one ExtProd (L = 2 with cts[0] = 0), short chains, the 128-step chain of the
16 GB geometry and the 256-step chain of the 64 GB one, and edge values
(zeros and q - 1 everywhere)."""
import numpy as np
import pytest

from oracle_lib import N, QS

pytestmark = pytest.mark.gpu


def _poly2(rng):
    return np.concatenate([rng.integers(0, QS[0], N, dtype=np.uint64), rng.integers(0, QS[1], N, dtype=np.uint64)])


def _inputs(L, seed):
    rng = np.random.default_rng(seed)
    rgsw = np.concatenate([_poly2(rng) for _ in range(8)])            # [4 parts][digit][limb][N]
    cts = np.concatenate([np.concatenate([_poly2(rng), _poly2(rng)]) for _ in range(L)])
    return rgsw, cts


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_ext_prod_matches_reference(ref, variant):
    import inspire_b200 as ib
    rgsw, cts = _inputs(2, 11 + variant)
    cts[: 4 * N] = 0                                  # acc = ExtProd(rgsw, ct[1]) + 0
    want = ref.ext_prod(rgsw, cts[4 * N:])
    assert (ib.horner_eval(rgsw, cts, 2, variant) == want).all()


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("L", [1, 3, 8, 128, 256])
def test_horner_chain_matches_reference(ref, variant, L):
    import inspire_b200 as ib
    rgsw, cts = _inputs(L, 100 * L + variant)
    assert (ib.horner_eval(rgsw, cts, L, variant) == ref.horner(rgsw, cts, L)).all()


@pytest.mark.parametrize("fill", ["zero", "max"])
def test_horner_edge_values(ref, fill):
    import inspire_b200 as ib
    L = 8
    rgsw, cts = _inputs(L, 5)
    if fill == "zero":
        cts[:] = 0
    else:
        for arr in (rgsw, cts):
            a = arr.reshape(-1, N)
            for r in range(a.shape[0]):
                a[r] = QS[r & 1] - 1                 # rows alternate limbs in both layouts
    want = ref.horner(rgsw, cts, L)
    for v in (0, 1, 2):
        assert (ib.horner_eval(rgsw, cts, L, v) == want).all(), v
