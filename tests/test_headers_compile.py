"""The public headers compile as their consumers compile them: the C ABI
header as C99 (FFI bindings, the reference's C callers) and the C++ protocol
header as C++17, both with warnings as errors.  CPU only (syntax check)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


@pytest.mark.parametrize("lang,std,src", [
    ("c", "c99", '#include "inspire_b200.h"\n'
                 "int main(void) { ipir_serve_config c = {0}; ipir_query_view v = {0};\n"
                 "  (void)v; return c.scan_segments; }\n"),
    ("c++", "c++17", '#include "inspire_b200.hpp"\nint main() { return 0; }\n'),
])
def test_public_header_compiles(tmp_path, lang, std, src):
    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("no host compiler")
    f = tmp_path / ("probe.c" if lang == "c" else "probe.cpp")
    f.write_text(src)
    cmd = [cc, f"-std={std}", "-Wall", "-Wextra", "-Werror", "-fsyntax-only", "-I", INC, str(f)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
