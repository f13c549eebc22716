"""End-to-end parity of the CUDA server through the C ABI: precomputed
tensors and encoded DB bit-exact against the oracle, every response
bit-exact against the oracle, and the reference client's extract()
recovering the queried entry (reference tests/test_e2e_gpu.cu)."""
import numpy as np
import pytest

from cases import get_case
from oracle_lib import N, PRE_A, PRE_D, PRE_F

pytestmark = pytest.mark.gpu

CASES = {
    "small": [0, 42, 100, 200, 255],
    "medium": [0, 42, 1000, 100000, 262143],
    "cfg1": [0, 1, 777, 40000, 65535],
}


@pytest.fixture(scope="module", params=list(CASES))
def served(request):
    import inspire_b200 as ib
    c = get_case(request.param)
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=c.db_rows_arg, max_batch=4, crs_seed=c.seed)
    yield request.param, c, srv
    srv.close()


def test_params_match_reference_setup(served):
    _, c, srv = served
    p = srv.params
    assert [p[k] for k in ("n_entries", "entry_bytes", "db_rows", "db_cols", "n_packed",
                           "interp_d", "num_cts")] == c.geom
    assert p["seed"] == c.seed and p["ring_n"] == N and p["d_eff"] == 2


def test_encoded_db_matches_oracle(served):
    _, c, srv = served
    dbe, _ = c.pre
    rows = min(c.R, 64)
    got = srv.export_db(0, rows)
    assert (got == dbe[: rows * c.C]).all()
    got = srv.export_db(c.R - rows, rows)
    assert (got == dbe[(c.R - rows) * c.C:]).all()


def test_precomp_matches_oracle(served):
    _, c, srv = served
    _, (pa, pdp, pdm, pdf) = c.pre
    for g in sorted({0, c.G - 1}):
        a, dp, dm, df = srv.export_precomp(g)
        assert (a == pa[g * PRE_A:(g + 1) * PRE_A]).all(), f"a group {g}"
        assert (df == pdf[g * PRE_F:(g + 1) * PRE_F]).all(), f"D_final group {g}"
        assert (dp == pdp[g * PRE_D:(g + 1) * PRE_D]).all(), f"D_plus group {g}"
        assert (dm == pdm[g * PRE_D:(g + 1) * PRE_D]).all(), f"D_minus group {g}"


def test_answers_bit_exact_and_extract(served):
    name, c, srv = served
    for k, idx in enumerate(CASES[name]):
        q, st = c.query(idx, 1000 + k)
        got = srv.answer(q)
        exp = c.oracle_answer(q)
        assert (got == exp).all(), f"{name} idx={idx}: response differs from the oracle"
        assert (st.extract(got) == c.expected_slots(idx)).all(), f"{name} idx={idx}: extract"


def test_batch_equals_singles(served):
    name, c, srv = served
    idxs = CASES[name][:4]
    qs = [c.query(i, 2000 + k)[0] for k, i in enumerate(idxs)]
    singles = np.stack([srv.answer(q) for q in qs])
    batch = srv.answer_batch(qs)
    assert (batch == singles).all()
