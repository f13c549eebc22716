"""Exact mat-vec paths: the tcgen05 int8 kernel and the CUDA-core kernel give
bit-identical responses, equal to the oracle, across batch sizes (one and
two tensor-core passes), K-chunked accumulation and partial batches."""
import os

import numpy as np
import pytest

from cases import get_case

pytestmark = pytest.mark.gpu


def make_server(c, mode, max_batch):
    import inspire_b200 as ib
    old = os.environ.get("IPB_MATVEC")
    os.environ["IPB_MATVEC"] = mode
    try:
        return ib.Server(c.n_entries, c.w, c.db, db_rows=c.db_rows_arg, max_batch=max_batch, crs_seed=c.seed)
    finally:
        if old is None:
            del os.environ["IPB_MATVEC"]
        else:
            os.environ["IPB_MATVEC"] = old


@pytest.mark.parametrize("name", ["batch", "cfg1"])
def test_tensor_core_matvec_matches_cuda_core_and_oracle(name):
    c = get_case(name)
    rng = np.random.default_rng(11)
    idxs = [int(x) for x in rng.integers(0, c.n_entries, 40)]
    qs = [c.query(i, 7000 + k)[0] for k, i in enumerate(idxs)]
    tc = make_server(c, "tc", 40)
    simt = make_server(c, "simt", 40)
    try:
        for n in (1, 2, 5, 17, 32, 40):
            a = tc.answer_batch(qs[:n])
            b = simt.answer_batch(qs[:n])
            assert (a == b).all(), f"{name}: tcgen05 and CUDA-core responses differ at batch {n}"
        for i in (0, 39):
            assert (a[i] == c.oracle_answer(qs[i])).all(), i
    finally:
        tc.close()
        simt.close()
