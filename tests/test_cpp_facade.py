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
