"""The CUDA server against the committed golden fixtures (tests/golden/*.npz,
responses of the reference's own GPU server): the packed query answered
through ipir_b200_answer_wire gives the fixture's packed and compressed
response bytes, and the flat answer packs to the same bytes.  Inputs are
rebuilt from the fixture's seeds; nothing of the reference is read."""
import glob
import hashlib
import os
import sys

import numpy as np
import pytest

from oracle_lib import crs_seed_from

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import wire  # noqa: E402

FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_server_reproduces_golden(path):
    import inspire_b200 as ib
    f = np.load(path)
    g = [int(x) for x in f["geom"]]
    db = wire.splitmix_db(g[2] * g[3], int(f["db_seed"]))
    assert hashlib.sha256(db.tobytes()).hexdigest() == str(f["db_sha256"])
    srv = ib.Server(int(f["n_entries"]), int(f["w"]), db, db_rows=int(f["db_rows"]), max_batch=2,
                    crs_seed=crs_seed_from(int(f["crs"])))
    try:
        qp = np.ascontiguousarray(f["query_packed"])
        two = np.concatenate([qp, qp])
        got_p = srv.answer_wire(two, 2, ib.RESP_PACKED)
        got_c = srv.answer_wire(two, 2, ib.RESP_COMPRESSED)
        for k in range(2):
            assert (got_p[k] == f["resp_packed"]).all(), k
            assert (got_c[k] == f["resp_compressed"]).all(), k
        flat = srv.answer(wire.unpack_query(qp, g[2]))
        assert (wire.pack_response(flat, g[6]) == f["resp_packed"]).all()
    finally:
        srv.close()
