"""Server checkpoints on the GPU: a handle restored from its saved state (no
raw DB, no preprocessing) answers bit-identically to the handle that saved
it (tolerance 0), and a flipped byte in any section fails the device-side
checksum on load."""
import os

import numpy as np
import pytest

from cases import get_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,idx", [("small", [0, 255]), ("medium", [7, 262143])])
def test_restored_handle_answers_identically(name, idx, tmp_path):
    import inspire_b200 as ib
    c = get_case(name)
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=2, crs_seed=c.seed)
    path = tmp_path / f"{name}.ckpt"
    L = ib.library_handle()
    rows_before = np.zeros((2, c.C), np.uint16)
    try:
        srv.save(path)
        qs, sts = zip(*[c.query(i, 9100 + k) for k, i in enumerate(idx)])
        want = srv.answer_batch(list(qs))
        assert L.ipir_b200_export_db(srv._h, c.R - 2, 2, rows_before.ctypes.data_as(ib.u16p)) == 0
    finally:
        srv.close()
    back = ib.Server.load(path, max_batch=2)
    try:
        assert back.params == srv.params
        got = back.answer_batch(list(qs))
        assert (got == want).all()
        assert (back.answer(qs[0]) == want[0]).all()
        for k, st in enumerate(sts):
            assert (st.extract(got[k]) == c.expected_slots(idx[k])).all()
        rows = np.zeros((2, c.C), np.uint16)           # the encoded DB came back as saved
        assert L.ipir_b200_export_db(back._h, c.R - 2, 2, rows.ctypes.data_as(ib.u16p)) == 0
        assert (rows == rows_before).all()
    finally:
        back.close()


def test_corrupted_sections_fail_the_checksum(tmp_path):
    import inspire_b200 as ib
    c = get_case("small")
    srv = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=1, crs_seed=c.seed)
    path = tmp_path / "small.ckpt"
    srv.save(path)
    srv.close()
    raw = bytearray(path.read_bytes())
    R, Cc = c.R, c.C
    sizes = [R * Cc * 2, 2 * 2048 * 4, 2 * 2048 * 4 * 1 * 4096, 2 * 2 * 2048 * 4]
    assert len(raw) == 256 + sum(sizes)
    starts = np.cumsum([256] + sizes[:-1])
    for k, label in enumerate(["DB", "a", "D byte planes", "D_final"]):
        bad = bytearray(raw)
        bad[int(starts[k]) + sizes[k] // 2] ^= 0x01
        f = tmp_path / f"bad{k}.ckpt"
        f.write_bytes(bad)
        with pytest.raises(ib.InspireError, match=f"checksum mismatch \\({label}\\)"):
            ib.Server.load(f, max_batch=1)
        os.remove(f)


def test_checkpoint_as_next_generation(tmp_path):
    """A database refreshed offline, saved, and restored from its checkpoint
    replaces the live generation of a serving loop: after the swap every
    response is the restored handle's, bit-identical to the handle that was
    saved."""
    import inspire_b200 as ib
    c = get_case("medium")
    live = ib.Server(c.n_entries, c.w, c.db, db_rows=2048, max_batch=2, crs_seed=c.seed)
    fresh = ib.Server(c.n_entries, c.w, ib.fill_db(c.R * c.C, 91), db_rows=2048, max_batch=2, crs_seed=c.seed)
    path = tmp_path / "next.ckpt"
    qs = [c.query(i, 9200 + k)[0] for k, i in enumerate([3, 200000, 3])]
    try:
        fresh.save(path)
        want_new = [fresh.answer(q) for q in qs]
        want_old = [live.answer(q) for q in qs]
    finally:
        fresh.close()
    restored = ib.Server.load(path, max_batch=2)
    loop = ib.ServeLoop([live], max_batch=2, lanes_per_db=2, queue_slots=16, autotune=False)
    try:
        r = np.zeros(ib.response_u64s(live.params), np.uint64)
        loop.wait(loop.submit(0, qs[0]), out=r)
        assert (r == want_old[0]).all()
        loop.replace_db(0, restored)
        for q, w in zip(qs, want_new):
            loop.wait(loop.submit(0, q), out=r)
            assert (r == w).all()
    finally:
        loop.close()
        restored.close()
        live.close()
