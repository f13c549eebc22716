"""Every struct of the C ABI header and its ctypes mirror in the Python
package agree field by field: names, order, per-field sizes and the whole
struct's size and alignment.  A field added to the header but not to the
mirror (or the other way round) would make the library read past the
caller's struct.  Runs on the CPU (the header is parsed as text)."""
import ctypes as C
import os
import re

import pytest

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "inspire_b200.h")

MIRRORS = {
    "ipir_params": "IpirParams",
    "ipir_caps": "IpirCaps",
    "ipir_query_view": "IpirQueryView",
    "ipir_matvec_opts": "IpirMatvecOpts",
    "ipir_serve_schedule": "IpirSchedule",
    "ipir_serve_config": "IpirServeConfig",
    "ipir_serve_counters": "IpirServeCounters",
    "ipir_serve_batch_record": "IpirServeBatchRecord",
}

C_SIZES = {"size_t": 8, "int": 4, "double": 8, "float": 4, "uint8_t": 1, "uint16_t": 2, "uint32_t": 4,
           "uint64_t": 8, "int32_t": 4, "int64_t": 8}


def header_structs():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    out = {}
    for body, name in re.findall(r"typedef struct\s*\{(.*?)\}\s*(\w+)\s*;", text, flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            m = re.match(r"^(?:const\s+)?(\w+)\s*(\*?)\s*(.*)$", decl)
            assert m, decl
            base, ptr, names = m.group(1), m.group(2), m.group(3)
            for nm in names.split(","):
                nm = nm.strip()
                star = ptr or nm.startswith("*")
                nm = nm.lstrip("*").strip()
                arr = re.match(r"^(\w+)\s*\[(\d+)\]$", nm)
                count = int(arr.group(2)) if arr else 1
                nm = arr.group(1) if arr else nm
                size = 8 if star else C_SIZES[base]
                fields.append((nm, size * count, 8 if star else C_SIZES[base]))
        out[name] = fields
    return out


def c_layout(fields):
    off, align = 0, 1
    for _, size, a in fields:
        off = (off + a - 1) // a * a + size
        align = max(align, a)
    return (off + align - 1) // align * align, align


@pytest.mark.parametrize("cname", sorted(MIRRORS))
def test_ctypes_mirror_matches_header(cname):
    import inspire_b200 as ib
    structs = header_structs()
    assert cname in structs, f"{cname} not found in the header"
    fields = structs[cname]
    py = getattr(ib, MIRRORS[cname])
    assert [f[0] for f in py._fields_] == [f[0] for f in fields], cname
    for (name, ctype), (_, size, _) in zip(py._fields_, fields):
        assert C.sizeof(ctype) == size, (cname, name, C.sizeof(ctype), size)
    size, align = c_layout(fields)
    assert C.sizeof(py) == size, (cname, C.sizeof(py), size)
    assert C.alignment(py) == align, cname


def test_every_header_struct_has_a_mirror():
    assert sorted(header_structs()) == sorted(MIRRORS)
