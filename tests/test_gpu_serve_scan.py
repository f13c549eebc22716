"""Serving loop in cyclic-scan mode (ipir_serve_config.scan_segments): the
DB pass runs as column segments and the tensor pass as (limb, slot)
segments in rotation, requests join at the next segment, and a query's
partial results stay under its lane slot until its last segment.  Every
response must be bit-identical to the plain single answer of the same query
(tolerance 0) whichever segment it joined at and whatever shared its
segments; responses decrypt through the reference client's extract() to the
queried entry.  A segment count that does not split the columns into
multiples of 128 leaves the database on lane batches."""
import random
import time

import numpy as np
import pytest

from cases import get_case

pytestmark = pytest.mark.gpu

N_REQ = 20


@pytest.fixture(scope="module")
def env():
    import inspire_b200 as ib
    c = get_case("g128")
    assert c.G == 128
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=8, crs_seed=c.seed)
    rng = np.random.default_rng(31)
    idxs = [int(x) for x in rng.integers(0, c.n_entries, N_REQ)]
    idxs[3] = idxs[4]   # the same entry twice, fresh keys
    qs, sts = [], []
    for k, idx in enumerate(idxs):
        q, st = c.query(idx, 9100 + k)
        qs.append(q)
        sts.append(st)
    singles = [srv.answer(q) for q in qs]
    yield ib, c, srv, idxs, qs, sts, singles
    srv.close()


def _serve(ib, srv, qs, rng, gaps, **cfg):
    loop = ib.ServeLoop([srv], **cfg)
    try:
        tickets = []
        for q in qs:
            tickets.append(loop.submit(0, q))
            if gaps and rng.random() < 0.5:   # later requests join at later segments
                time.sleep(rng.uniform(0.0, 0.003))
        out = []
        for t in tickets:
            r = np.zeros(ib.response_u64s(srv.params), np.uint64)
            assert loop.wait(t, out=r, timeout=60.0) >= 0.0
            out.append(r)
        stats = loop.stats()
        info = loop.db_info(0)
        trace = loop.trace()
    finally:
        loop.close()
    return out, stats, info, trace


@pytest.mark.parametrize("segments,gaps", [(4, True), (2, True), (4, False)])
def test_scan_equals_singles(env, segments, gaps):
    ib, c, srv, idxs, qs, sts, singles = env
    out, stats, info, trace = _serve(ib, srv, qs, random.Random(segments), gaps, max_batch=8, queue_slots=64,
                                     autotune=False, scan_segments=segments)
    for i in range(N_REQ):
        assert (out[i] == singles[i]).all(), (segments, i)
    assert stats["completed"] == N_REQ and stats["failed"] == 0 and stats["queued"] == 0
    assert stats["batched_queries"] == N_REQ and stats["free_slots"] == 64
    assert 1 <= stats["max_batch_seen"] <= 8      # a group holds at most the lane's 8 slots
    assert info["lanes"] == 1 and info["max_batch"] == 8
    assert sum(t["count"] for t in trace) == N_REQ and not any(t["failed"] for t in trace)
    if not gaps:
        assert stats["batches"] >= 3               # 20 requests at once: groups of <= 8 slots
    for i in (0, 3, 4, N_REQ - 1):
        assert (sts[i].extract(out[i]) == c.expected_slots(idxs[i])).all(), i
    assert not (out[3] == out[4]).all()


def test_segments_that_do_not_split_fall_back_to_lanes(env):
    ib, c, srv, idxs, qs, sts, singles = env
    out, stats, info, _ = _serve(ib, srv, qs[:6], random.Random(5), True, max_batch=4, lanes_per_db=2,
                                 queue_slots=16, autotune=False, scan_segments=3)
    assert info["lanes"] == 2
    for i in range(6):
        assert (out[i] == singles[i]).all(), i


@pytest.mark.parametrize("threshold_ms,scan", [("0", True), ("1000", False)])
def test_auto_scan_choice(env, monkeypatch, threshold_ms, scan):
    """scan_segments < 0: the loop times each database's plain answer at
    create and serves it by cyclic scan from a threshold (2 ms, here moved
    by IPB_SCAN_AUTO_MS to 0 and to 1000 ms) and by lane batches below;
    either way every response equals the plain single answer."""
    ib, c, srv, idxs, qs, sts, singles = env
    monkeypatch.setenv("IPB_SCAN_AUTO_MS", threshold_ms)
    out, stats, info, _ = _serve(ib, srv, qs[:8], random.Random(17), True, max_batch=8, lanes_per_db=2,
                                 queue_slots=32, autotune=False, scan_segments=-1)
    assert info["lanes"] == (1 if scan else 2)
    for i in range(8):
        assert (out[i] == singles[i]).all(), (threshold_ms, i)
    assert stats["failed"] == 0


def test_scan_packed_slots_and_generation_swap():
    """G = 4: the tensor pass packs eight (limb, slot) items into one 128-row
    tile, so each segment's slot range is whole packed items.  Scan responses
    equal single answers, a duplicate index with fresh keys stays distinct,
    and a generation swap replaces the database between rotations: after it
    every response is the new handle's."""
    import inspire_b200 as ib
    c = get_case("medium")
    live = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=4, crs_seed=c.seed)
    nxt = ib.Server(c.n_entries, c.w, ib.fill_db(c.R * c.C, 91), db_rows=2048, max_batch=4, crs_seed=c.seed)
    idx = [3, 200000, 3, 77, 262143, 1000]
    qs = [c.query(i, 9300 + k) for k, i in enumerate(idx)]
    try:
        old = [live.answer(q) for q, _ in qs]
        new = [nxt.answer(q) for q, _ in qs]
        loop = ib.ServeLoop([live], max_batch=4, queue_slots=16, autotune=False, scan_segments=4)
        try:
            assert loop.db_info(0)["lanes"] == 1
            r = np.zeros(ib.response_u64s(live.params), np.uint64)
            for want in (old, new):
                ts = [loop.submit(0, q) for q, _ in qs]
                for k, t in enumerate(ts):
                    loop.wait(t, out=r, timeout=60.0)
                    assert (r == want[k]).all(), k
                    if want is old and k in (0, 2):
                        assert (qs[k][1].extract(r) == c.expected_slots(idx[k])).all(), k
                if want is old:
                    loop.replace_db(0, nxt)
            assert loop.stats()["completed"] == 2 * len(qs)
        finally:
            loop.close()
        assert not (old[0] == old[2]).all()
    finally:
        live.close()
        nxt.close()


def test_close_with_requests_in_the_rotation(env):
    """Destroying the loop right after submitting: the rotation runs its
    admitted requests to the end (requests still waiting fail), and destroy
    returns.  A watchdog thread bounds the wait so a regression fails the
    test instead of hanging the run."""
    import threading
    ib, c, srv, idxs, qs, sts, singles = env
    loop = ib.ServeLoop([srv], max_batch=8, queue_slots=64, autotune=False, scan_segments=4)
    for q in qs:
        loop.submit(0, q)
    done = threading.Event()

    def close():
        loop.close()
        done.set()

    th = threading.Thread(target=close, daemon=True)
    th.start()
    assert done.wait(60.0), "ipir_serve_destroy did not return"
    # the handle still answers on its own afterwards
    assert (srv.answer(qs[0]) == singles[0]).all()
