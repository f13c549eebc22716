"""The oracle and the wire-format restatement against the committed golden
fixtures (tests/golden/*.npz): responses of the reference's own GPU server
to reference-client queries, generated by tests/golden/make_golden.py.
Neither the reference sources nor its build are needed here."""
import glob
import hashlib
import os
import sys

import numpy as np
import pytest

from oracle_lib import Oracle, crs_seed_from

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import wire  # noqa: E402

FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def load(path):
    f = np.load(path)
    g = [int(x) for x in f["geom"]]
    db = wire.splitmix_db(g[2] * g[3], int(f["db_seed"]))
    assert hashlib.sha256(db.tobytes()).hexdigest() == str(f["db_sha256"])
    return f, g, db


def test_fixtures_present():
    assert len(FIXTURES) >= 2


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(p)[:-4] for p in FIXTURES])
def test_oracle_reproduces_reference_server(path):
    f, g, db = load(path)
    _, _, R, Cc, G, D, ncts = g
    o = Oracle()
    dbe, pre = o.preprocess(crs_seed_from(int(f["crs"])), db, R, Cc, D)
    q = wire.unpack_query(f["query_packed"], R)
    assert (wire.pack_query(q, R) == f["query_packed"]).all()
    resp = o.answer(dbe, R, Cc, D, pre, q)
    assert (wire.pack_response(resp, ncts) == f["resp_packed"]).all()
    assert (wire.unpack_response(f["resp_packed"], ncts) == resp).all()
    assert (wire.compress_response(resp, ncts, o.ntt_inverse) == f["resp_compressed"]).all()
    # the entry the client decoded sits at the queried index of the rebuilt DB
    w, idx = g[1], int(f["idx"])
    cpe = (w * 8 + 14) // 15
    want = [db[(idx % R) * Cc + (idx // R) * cpe + k] for k in range(cpe)]
    assert (f["slots"] == np.array(want, np.uint16)).all()


@pytest.mark.parametrize("path", FIXTURES[:1], ids=["codecs_vs_client_library"])
def test_wire_restatement_matches_client_library(path):
    """The numpy codecs against the reference client library compiled from
    its sources (skipped where that build is absent)."""
    try:
        from oracle_lib import RefLib, ref_params
        r = RefLib()
    except (FileNotFoundError, OSError):
        pytest.skip("reference client library not built")
    f, g, _ = load(path)
    p = ref_params(g, (g[0], g[1]), crs_seed_from(int(f["crs"])))
    q = wire.unpack_query(f["query_packed"], g[2])
    assert (r.wire(p, "ipir_query_pack", q, "ipir_query_packed_bytes") == f["query_packed"]).all()
    resp = wire.unpack_response(f["resp_packed"], g[6])
    assert (r.wire(p, "ipir_response_compress", resp, "ipir_response_compressed_bytes") == f["resp_compressed"]).all()
