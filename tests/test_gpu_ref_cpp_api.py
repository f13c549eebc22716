"""The reference's C++ server API on its own types (src/gpu_protocol.h:44-78):
one consumer program, written only against the reference's headers
(tests/cpp/ref_consumer.cpp), built unchanged against this project's
libinspire_b200_refapi.so and against the reference's own GPU library,
runs setup -> gpu_preprocess -> gpu_setup_server -> query() -> gpu_answer ->
extract() (every entry recovered), gpu_answer_batch == singles (a repeated
index with fresh keys included), caps and free, on the Medium and Batch
geometries of the reference's tests and on setup(2^25, 30)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(REPO, "oracle", "_ref")


@pytest.mark.parametrize("impl", ["b200", "refgpu"])
@pytest.mark.parametrize("geom", [("262144", "120", "2048", "4"), ("524288", "120", "2048", "8"),
                                  (str(1 << 25), "30", "0", "3")])
def test_reference_cpp_consumer_runs_unchanged(impl, geom):
    exe = os.path.join(BIN, f"ref_consumer_{impl}")
    if not os.path.exists(exe):
        pytest.skip("consumer not built (needs the reference's headers: make -C oracle ref_consumer REF=...)")
    r = subprocess.run([exe, *geom], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.startswith("ok"), (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
