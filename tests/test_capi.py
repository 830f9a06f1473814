"""The C ABI library loads without a GPU and exports every symbol include/htcuda.h declares."""
import os
import re

import pytest

from hypertrace_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(htc_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = _declared("htcuda.h")
    assert "htc_render" in names and "htc_render_passes" in names and "htc_extract_gamma_pack" in names


def test_library_exports_every_declared_symbol(built):
    lib = _lib.lib()
    for name in _declared("htcuda.h"):
        assert hasattr(lib, name), f"libhtcuda.so does not export {name}"


def test_binding_covers_header(built):
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(_declared("htcuda.h")) <= bound


def test_errors_without_device(built):
    """Argument checks fail loudly with a message (no device needed for these)."""
    import ctypes
    h = ctypes.c_void_p()
    rc = _lib.lib().htc_program_create(99, 4, 32, 0, 0, ctypes.byref(h))
    assert rc == _lib.HTC_ERR_UNSUPPORTED
    assert b"recipe" in _lib.lib().htc_last_error()
    rc = _lib.lib().htc_program_create(1, 0, 32, 0, 0, ctypes.byref(h))
    assert rc == _lib.HTC_ERR_INVALID
    rc = _lib.lib().htc_program_create(3, 4, 32, 1, 0, ctypes.byref(h))   # double_support: HY / EU recipes only
    assert rc == _lib.HTC_ERR_UNSUPPORTED
    assert b"double_support" in _lib.lib().htc_last_error()
    rc = _lib.lib().htc_program_create(1, 4, 32, 0, 4, ctypes.byref(h))   # no such flag bit
    assert rc == _lib.HTC_ERR_INVALID
    assert b"flags" in _lib.lib().htc_last_error()
    rc = _lib.lib().htc_render(None, 4, 4, None, 0, None, None, None)
    assert rc == _lib.HTC_ERR_INVALID


def test_flag_values_match_header():
    """The Python mirror's flag bits are the header's."""
    text = open(os.path.join(ROOT, "include", "htcuda.h")).read()
    flags = dict(re.findall(r"#define (HTC_FLAG_\w+) (\d+)u", text))
    assert int(flags["HTC_FLAG_JITTER_YX"]) == _lib.HTC_FLAG_JITTER_YX
    assert int(flags["HTC_FLAG_NO_SORT"]) == _lib.HTC_FLAG_NO_SORT


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "nope.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.lib()


def test_newer_entry_points_reject_bad_arguments_without_device(built):
    """The wavefront, batch-reservation and seed-fill entry points check their arguments
    before touching a device."""
    lib = _lib.lib()
    assert lib.htc_render_wavefront(None, 4, 4, None, 0, None, None, 1, None, None) == _lib.HTC_ERR_INVALID
    assert lib.htc_render_passes(None, 4, 4, None, 0, None, None, 1, None, None) == _lib.HTC_ERR_INVALID
    assert lib.htc_batch_reserve(None, 1024, 8, None) == _lib.HTC_ERR_INVALID
    assert b"batch" in lib.htc_last_error()
    assert lib.htc_fill_seeds(None, 5, 0, 0, None) == _lib.HTC_ERR_INVALID
    assert lib.htc_fill_seeds(None, 0, 0, 0, None) == _lib.HTC_OK   # nothing to fill
