"""Server checkpoint files (ipir_b200_save_server / ipir_b200_load_server):
every malformed file is rejected from its header and size alone, before any
device work, so these run without a GPU."""
import struct

import pytest

N = 2048


def _header(geom, seed=bytes(64), sizes=None, magic=b"IPIRB200", version=1, hbytes=256):
    n_entries, w, R, Cc, G, D, ncts = geom
    if sizes is None:
        sizes = [R * Cc * 2, G * 2 * N * 4, 2 * N * 4 * G * 4096, G * 2 * 2 * N * 4]
    h = magic + struct.pack("<II", version, hbytes) + struct.pack("<7Q", *geom) + seed
    h += struct.pack("<4Q", *sizes) + struct.pack("<4Q", 0, 0, 0, 0)
    return h + bytes(256 - len(h)), sizes


@pytest.fixture(scope="module")
def ib():
    import inspire_b200
    return inspire_b200


@pytest.fixture(scope="module")
def small_geom(ib):
    p = ib.setup(256, 120, 2048)
    return [p["n_entries"], p["entry_bytes"], p["db_rows"], p["db_cols"], p["n_packed"], p["interp_d"],
            p["num_cts"]]


def _load_error(ib, path):
    with pytest.raises(ib.InspireError) as e:
        ib.Server.load(str(path), max_batch=1)
    return str(e.value)


def test_missing_and_foreign_files(ib, tmp_path):
    assert "cannot open" in _load_error(ib, tmp_path / "none.ckpt")
    f = tmp_path / "foreign.ckpt"
    f.write_bytes(b"\x7fELF" + bytes(300))
    assert "magic" in _load_error(ib, f)
    f.write_bytes(b"IPIRB200")
    assert "short header" in _load_error(ib, f)


def test_header_checks(ib, tmp_path, small_geom):
    f = tmp_path / "bad.ckpt"
    head, sizes = _header(small_geom, version=2)
    f.write_bytes(head)
    assert "version" in _load_error(ib, f)
    bad = list(small_geom)
    bad[1] = 32                                   # setup() rejects w = 32
    f.write_bytes(_header(bad)[0])
    assert "geometry rejected" in _load_error(ib, f)
    bad = list(small_geom)
    bad[3] *= 2                                   # db_cols not what setup() gives
    f.write_bytes(_header(bad)[0])
    assert "inconsistent" in _load_error(ib, f)
    head, sizes = _header(small_geom, sizes=[1, 2, 3, 4])
    f.write_bytes(head)
    assert "section size" in _load_error(ib, f)


def test_truncated_and_oversized(ib, tmp_path, small_geom):
    head, sizes = _header(small_geom)
    f = tmp_path / "short.ckpt"
    f.write_bytes(head + bytes(1000))
    assert "truncated" in _load_error(ib, f)
    with open(f, "wb") as o:                      # one byte more than the sections
        o.write(head)
        o.truncate(256 + sum(sizes) + 1)
    assert "oversized" in _load_error(ib, f)


def test_null_arguments(ib, tmp_path):
    L = ib.library_handle()
    assert L.ipir_b200_save_server(None, str(tmp_path / "x").encode()) == 1
    p = ib.IpirParams()
    assert L.ipir_b200_load_server(None, 1, p) is None
    assert L.ipir_b200_load_server(str(tmp_path / "x").encode(), 0, p) is None
