"""The C++ facade (include/paulib_b200.hpp): it compiles and links against
the in-tree library here; on a GPU its known-answer program runs and passes
(tests/cpp/facade_test.cpp restates PauliSumTests.cpp assertions)."""
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "tests", "cpp", "build.sh")


def _build(out):
    r = subprocess.run(["sh", BUILD, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]


def test_facade_compiles_and_links():
    with tempfile.TemporaryDirectory() as d:
        _build(os.path.join(d, "facade_test"))


@pytest.mark.gpu
def test_facade_known_answers(cuda):
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "facade_test")
        _build(exe)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
        assert "0 failed" in r.stdout


# The reference's own GPU host wrapper (include/gpu/GpuPauliSum.h) linked
# against this library.  It needs the reference headers to compile, so it is
# built where they are (__graft_entry__.build(), or the test below) into
# tests/cpp/_build/, and the GPU test runs the built binary.
WRAPPER = os.path.join(ROOT, "tests", "cpp", "_build", "gpu_wrapper_test")
REF_DIR = os.environ.get("PAULIB_REFERENCE_DIR", "/root/reference")


def test_reference_wrapper_compiles_against_library():
    if not os.path.isdir(os.path.join(REF_DIR, "include", "gpu")):
        pytest.skip("reference headers not present (the GPU test uses the prebuilt binary)")
    os.makedirs(os.path.dirname(WRAPPER), exist_ok=True)
    r = subprocess.run(["sh", os.path.join(ROOT, "tests", "cpp", "build_wrapper.sh"), WRAPPER],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.mark.gpu
def test_reference_wrapper_runs_on_library(cuda):
    assert os.path.exists(WRAPPER), "tests/cpp/_build/gpu_wrapper_test not built (run build())"
    r = subprocess.run([WRAPPER], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "9 passed, 0 failed" in r.stdout
