"""The C-ABI library loads without a GPU and exports every symbol that
include/paulib_b200.h declares (no compute calls are made here)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "paulib_b200.h")) as fh:
        text = fh.read()
    return re.findall(r"^PL_API\s+[\w\s\*]*?\b((?:pl|launch_gpu)_\w+)\(", text, re.M)


def test_header_declares_the_reference_seam():
    syms = declared_symbols()
    # the two launchers of the reference's include/gpu/paulib_gpu_api.h
    assert "launch_gpu_mul_soa" in syms and "launch_gpu_commutator_soa" in syms
    assert len(syms) == len(set(syms))


def test_library_exports_every_declared_symbol():
    from paulib_b200 import _abi
    lib = _abi.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"not exported: {missing}"
    assert set(declared_symbols()) == set(_abi.EXPORTS)


def test_status_strings_without_gpu():
    from paulib_b200 import _abi
    lib = _abi.lib()
    assert lib.pl_status_string(0) == b"ok"
    assert lib.pl_status_string(_abi.PL_ERR_CAPACITY) == b"output capacity exceeded"
    assert lib.pl_version() >= 1


def test_invalid_arguments_are_reported_not_trapped():
    # Argument validation happens before any device work, so this runs on CPU.
    from paulib_b200 import _abi
    lib = _abi.lib()
    nb = ctypes.c_size_t()
    assert lib.pl_collate_workspace_size(0, 10, ctypes.byref(nb)) == _abi.PL_ERR_INVALID_ARG
    assert lib.pl_collate_workspace_size(17, 10, ctypes.byref(nb)) == _abi.PL_ERR_INVALID_ARG
    assert lib.pl_collate_workspace_size(4, 1000, ctypes.byref(nb)) == _abi.PL_OK
    assert nb.value > 1000
    # the void drop-in records the status instead of trapping (reference:
    # src/gpu/gpu_mul.cu:122-131 calls __builtin_trap())
    lib.launch_gpu_mul_soa(17, *([None] * 12), 1, 1, None)
    assert lib.pl_get_last_error() == _abi.PL_ERR_INVALID_ARG
    assert b"array_size" in lib.pl_last_error_message()
