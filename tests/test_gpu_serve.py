"""Serving loop (ipir_serve_*): continuous batching over two resident
databases of different geometry.  Every response must be bit-identical to
the plain single answer of the same query, alone vs in the mix (tolerance
0), whatever batch it landed in; graph replay and direct launches agree;
duplicate indices with fresh keys stay distinct and decrypt to the entry;
the request-slot and ticket codes behave as the header states."""
import random
import time

import numpy as np
import pytest

from cases import get_case

pytestmark = pytest.mark.gpu

IDX_A = [0, 7, 100, 65535, 262143, 12345, 0, 7]      # medium: 262144 entries, G = 4
IDX_B = [0, 42, 1000, 100000, 524287, 77777, 42, 42]  # batch: 524288 entries, G = 8


@pytest.fixture(scope="module")
def env():
    import inspire_b200 as ib
    ca, cb = get_case("medium"), get_case("batch")
    sa = ib.Server(ca.n_entries, ca.w, ca.db, db_rows=2048, max_batch=4, crs_seed=ca.seed)
    sb = ib.Server(cb.n_entries, cb.w, cb.db, db_rows=2048, max_batch=4, crs_seed=cb.seed)
    reqs = []   # (db, idx, flat query, client state)
    for k, idx in enumerate(IDX_A):
        q, st = ca.query(idx, 5000 + k)
        reqs.append((0, idx, q, st))
    for k, idx in enumerate(IDX_B):
        q, st = cb.query(idx, 6000 + k)
        reqs.append((1, idx, q, st))
    alone = [(sa if d == 0 else sb).answer(q) for d, _, q, _ in reqs]
    yield ca, cb, sa, sb, reqs, alone
    sa.close()
    sb.close()


def _run_mix(ib, servers, reqs, rng, **cfg):
    loop = ib.ServeLoop(servers, **cfg)
    try:
        order = list(range(len(reqs)))
        rng.shuffle(order)
        tickets = {}
        for j, i in enumerate(order):
            tickets[i] = loop.submit(reqs[i][0], reqs[i][2])
            if rng.random() < 0.3:           # gaps: later requests arrive while earlier ones run
                time.sleep(rng.uniform(0.0, 0.004))
        out = {}
        for i, t in tickets.items():
            r = np.zeros(ib.response_u64s(servers[reqs[i][0]].params), np.uint64)
            lat = loop.wait(t, out=r, timeout=30.0)
            assert lat >= 0.0
            out[i] = r
        stats = loop.stats()
        info = [loop.db_info(0), loop.db_info(1)]
    finally:
        loop.close()
    return out, stats, info


def test_mix_equals_alone(env):
    import inspire_b200 as ib
    ca, cb, sa, sb, reqs, alone = env
    out, stats, info = _run_mix(ib, [sa, sb], reqs, random.Random(11), max_batch=4, lanes_per_db=2,
                                queue_slots=32)
    for i in range(len(reqs)):
        assert (out[i] == alone[i]).all(), i
    assert stats["completed"] == len(reqs) and stats["failed"] == 0 and stats["queued"] == 0
    assert stats["batched_queries"] == len(reqs) and stats["free_slots"] == 32
    assert 1 <= stats["max_batch_seen"] <= 4
    for d in info:
        assert d["lanes"] == 2 and d["max_batch"] == 4
        for c, s in d["schedule"].items():
            assert s["matvec_tc"] in (0, 1) and s["horner_cluster"] in (0, 1, 2)
            assert (c + 1) // 2 <= s["tp_pass"] <= 4, (c, s)


def test_mix_bursts_batch_and_decrypt(env):
    """All requests at once: the loop must form multi-query batches; every
    response still equals its single answer, duplicate indices with fresh
    keys differ as ciphertexts and decrypt to the same entry."""
    import inspire_b200 as ib
    ca, cb, sa, sb, reqs, alone = env
    loop = ib.ServeLoop([sa, sb], max_batch=4, lanes_per_db=1, queue_slots=len(reqs), autotune=False)
    try:
        tickets = [loop.submit(d, q) for d, _, q, _ in reqs]
        outs = []
        for (d, _, _, _), t in zip(reqs, tickets):
            r = np.zeros(ib.response_u64s((sa if d == 0 else sb).params), np.uint64)
            loop.wait(t, out=r)
            outs.append(r)
        stats = loop.stats()
    finally:
        loop.close()
    assert stats["max_batch_seen"] > 1 and stats["batches"] < len(reqs)
    for i, (d, idx, _, st) in enumerate(reqs):
        assert (outs[i] == alone[i]).all(), i
        case = ca if d == 0 else cb
        assert (st.extract(outs[i]) == case.expected_slots(idx)).all(), i
    # IDX_A[0] == IDX_A[6]: same entry, fresh keys
    assert not (outs[0] == outs[6]).all()
    # one response against the oracle directly
    assert (outs[len(IDX_A)] == cb.oracle_answer(reqs[len(IDX_A)][2])).all()


def test_graphs_and_direct_launches_agree(env):
    """Direct launches with overlapping DB passes give the graph-replay results."""
    import inspire_b200 as ib
    ca, cb, sa, sb, reqs, alone = env
    out, stats, _ = _run_mix(ib, [sa, sb], reqs, random.Random(5), max_batch=3, lanes_per_db=2,
                             graphs=False, autotune=False, overlap_db_passes=True)
    for i in range(len(reqs)):
        assert (out[i] == alone[i]).all(), i
    assert stats["failed"] == 0


def test_tensor_pass_beside_matvec_in_graphs(env, monkeypatch):
    """Schedules that fork the tensor pass onto a second stream beside the
    mat-vec: captured into the per-batch-size graphs (and launched
    directly), every response equals the plain single answer."""
    import inspire_b200 as ib
    ca, cb, sa, sb, reqs, alone = env
    monkeypatch.setenv("IPB_TP_SMS", "48")
    for graphs in (True, False):
        out, stats, info = _run_mix(ib, [sa, sb], reqs, random.Random(11), max_batch=4, lanes_per_db=2,
                                    graphs=graphs, autotune=False, overlap_db_passes=not graphs)
        assert all(s["tp_sms"] == 48 for db in info for s in db["schedule"].values())
        for i in range(len(reqs)):
            assert (out[i] == alone[i]).all(), (graphs, i)
        assert stats["failed"] == 0


def test_chunked_horner_in_lanes(env, monkeypatch):
    """Schedules whose Horner chain trails the DB pass in group chunks run
    each lane batch as one pipeline (one graph per batch size, the DB-done
    event recorded inside it after the last chunk's finalize); with graph
    replay and with direct launches every response equals the plain single
    answer."""
    import inspire_b200 as ib
    ca, cb, sa, sb, reqs, alone = env
    monkeypatch.setenv("IPB_HCHUNKS", "8")
    monkeypatch.setenv("IPB_HORNER", "cl8")
    for graphs in (True, False):
        out, stats, info = _run_mix(ib, [sa, sb], reqs, random.Random(13), max_batch=4, lanes_per_db=2,
                                    graphs=graphs, autotune=False)
        assert all(s["hchunks"] == 8 for db in info for s in db["schedule"].values())
        for i in range(len(reqs)):
            assert (out[i] == alone[i]).all(), (graphs, i)
        assert stats["failed"] == 0


def test_slot_and_ticket_codes(env):
    import inspire_b200 as ib
    ca, cb, sa, sb, reqs, alone = env
    loop = ib.ServeLoop([sa], max_batch=2, lanes_per_db=1, queue_slots=3, autotune=False)
    try:
        v = ib.query_view_from_flat(sa.params, reqs[0][2])
        ts = []
        for _ in range(3):
            rc, t = loop.submit_view(0, v)
            assert rc == 0
            ts.append(t)
        rc, _ = loop.submit_view(0, v)
        assert rc == ib.SERVE_FULL                       # slots free only when collected
        rc, _ = loop.submit_view(1, v)
        assert rc == 1                                   # no such database
        r = np.zeros(ib.response_u64s(sa.params), np.uint64)
        for t in ts:
            loop.wait(t, out=r)
            assert (r == alone[0]).all()
        assert loop.poll(ts[0])[0] == ib.SERVE_UNKNOWN   # collected once already
        assert loop.poll(12345)[0] == ib.SERVE_UNKNOWN
        rc, t = loop.submit_view(0, v)                   # slots are free again
        assert rc == 0
        loop.wait(t, out=r)
        assert (r == alone[0]).all()
    finally:
        loop.close()


def test_handle_autotune_keeps_results(env):
    import inspire_b200 as ib
    ca, cb, sa, sb, reqs, alone = env
    sb.autotune()
    for c in range(1, 5):
        s = sb.schedule(c)
        assert s["matvec_tc"] in (0, 1) and s["horner_cluster"] in (0, 1, 2) and 1 <= s["tp_pass"] <= 4
        # sizes between the measured ones keep the measured split: at most two tensor passes
        assert s["tp_pass"] >= (c + 1) // 2, (c, s)
    qs = [q for d, _, q, _ in reqs if d == 1][:4]
    n0 = sb.launch_count()
    got = sb.answer_batch(qs)
    assert sb.launch_count() > n0
    want = np.stack([a for (d, _, _, _), a in zip(reqs, alone) if d == 1][:4])
    assert (got == want).all()


def test_generation_swap(env):
    """Replace a resident database by its next generation (same geometry,
    new contents) while the loop serves: before the swap every response is
    the old generation's, after it the new one's, and requests racing the
    swap get one of the two."""
    import threading
    import inspire_b200 as ib
    ca, cb, sa, sb, reqs, alone = env
    db2 = ib.fill_db(ca.R * ca.C, 77)
    sa2 = ib.Server(ca.n_entries, ca.w, db2, db_rows=2048, max_batch=4, crs_seed=ca.seed)
    try:
        qa = [q for d, _, q, _ in reqs if d == 0]
        new = [sa2.answer(q) for q in qa]
        old = [a for (d, _, _, _), a in zip(reqs, alone) if d == 0]
        assert not (new[0] == old[0]).all()
        loop = ib.ServeLoop([sa, sb], max_batch=4, lanes_per_db=2, queue_slots=64, autotune=False)
        try:
            r = np.zeros(ib.response_u64s(sa.params), np.uint64)
            t = loop.submit(0, qa[0])
            loop.wait(t, out=r)
            assert (r == old[0]).all()
            # requests racing the swap
            racing = [(i % len(qa), loop.submit(0, qa[i % len(qa)])) for i in range(12)]
            th = threading.Thread(target=loop.replace_db, args=(0, sa2))
            th.start()
            racing += [(i % len(qa), loop.submit(0, qa[i % len(qa)])) for i in range(12, 20)]
            th.join()
            for i, t in racing:
                loop.wait(t, out=r)
                assert (r == old[i]).all() or (r == new[i]).all(), i
            for i, q in enumerate(qa):
                t = loop.submit(0, q)
                loop.wait(t, out=r)
                assert (r == new[i]).all(), i
            # the other database is untouched
            t = loop.submit(1, reqs[len(qa)][2])
            loop.wait(t, out=r[: ib.response_u64s(sb.params)])
            assert (r[: ib.response_u64s(sb.params)] == alone[len(qa)]).all()
            st = loop.stats()
            assert st["failed"] == 0
        finally:
            loop.close()
    finally:
        sa2.close()


def test_hbm_budget_halves_batch_then_lanes_then_refuses(env):
    """Admission capacity is sized against the HBM budget at create: as the
    budget shrinks the loop first halves max_batch (64, 32, ... 1), then
    drops lanes (2 -> 1), then refuses to start (nothing is allocated per
    request afterwards, so no later check is needed); a loop sized down
    still answers bit-exactly."""
    import inspire_b200 as ib
    ca, cb, sa, sb, reqs, alone = env
    seen = []
    budget = 1 << 36
    while budget >= 1 << 16:
        try:
            loop = ib.ServeLoop([sa, sb], max_batch=64, lanes_per_db=2, hbm_budget_bytes=budget, graphs=False,
                                autotune=False)
        except ib.InspireError as e:
            assert "exceeds the HBM budget" in str(e)
            seen.append((0, 0))
            break
        info = loop.db_info(0)
        seen.append((info["max_batch"], info["lanes"]))
        if info["max_batch"] < 64 and not any(s[0] < 64 for s in seen[:-1]):   # the first shrunk loop answers
            d, _, q, _ = reqs[0]
            out = np.zeros_like(alone[0])
            loop.wait(loop.submit(d, q), out=out)
            assert (out == alone[0]).all()
        loop.close()
        budget //= 2
    assert seen[0] == (64, 2) and seen[-1] == (0, 0), seen
    order = [(-mb, -ln) for mb, ln in seen[:-1]]
    assert order == sorted(order), seen              # capacity only shrinks as the budget does
    lanes_at = [ln for mb, ln in seen[:-1]]
    assert 1 in lanes_at and all(mb == 1 for mb, ln in seen[:-1] if ln == 1), seen  # lanes drop only at batch 1
