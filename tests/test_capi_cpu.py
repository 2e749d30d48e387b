"""CPU-side checks of the C ABI: the library loads and exports every entry
point include/dpb200.h declares (no GPU calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dpb200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"DPB_API\s+[\w\s\*]+?\b(dpb_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("dpb_model_create", "dpb_nlist_build", "dpb_eval"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from deepmd_jax_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libdpb200.so not built")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for s in declared_symbols():
        assert hasattr(lib, s), s
    assert set(_lib.EXPORTED) <= set(declared_symbols())


def test_version_string():
    from deepmd_jax_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libdpb200.so not built")
    assert b"sm_100a" in _lib.load().dpb_version()


def test_jax_ffi_shim_build_target():
    """The jax.ffi shim's make target builds only where jaxlib's FFI headers
    exist and otherwise succeeds with a 'skipped' note (this image has no jax)."""
    import subprocess
    import importlib.util
    d = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "deepmd-jax_b200", "csrc", "jax_ffi")
    out = subprocess.run(["make", "-C", d], capture_output=True, text=True)
    assert out.returncode == 0
    if importlib.util.find_spec("jax") is None:
        assert "skipped: no jaxlib" in out.stdout
