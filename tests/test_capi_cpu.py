"""C-ABI checks that need no GPU: the library loads and exports every symbol
declared in include/rrtmg_b200.h; host-side helpers agree with the reference."""

from __future__ import annotations

import ctypes
import re

import pytest

from conftest import REPO


def _declared_symbols(header: str = "rrtmg_b200.h"):
    text = (REPO / "include" / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)  # declarations only, not comments
    return sorted(set(re.findall(r"\b(rrtmg_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = _declared_symbols()
    assert {"rrtmg_create", "rrtmg_lwrad", "rrtmg_swrad", "rrtmg_destroy"} <= set(names)


def test_library_exports_every_declared_symbol(pkg):
    from wrf_jax_b200 import _capi, build
    if not _capi.LIB_PATH.exists():
        build.build_library()
    lib = ctypes.CDLL(str(_capi.LIB_PATH))
    for header, exports in (("rrtmg_b200.h", _capi.EXPORTS), ("rrtmg_surrogate.h", _capi.SURROGATE_EXPORTS),
                            ("rrtmg_prologue.h", _capi.PROLOGUE_EXPORTS),
                            ("rrtmg_tendency.h", _capi.TENDENCY_EXPORTS),
                            ("rrtmg_tables.h", _capi.TABLES_EXPORTS),
                            ("rrtmg_xla_ffi.h", _capi.FFI_EXPORTS)):
        for name in _declared_symbols(header):
            assert hasattr(lib, name), name
        assert set(exports) == set(_declared_symbols(header))


@pytest.mark.parametrize("p_top,nk", [(5000.0, 44), (5000.0, 50), (1000.0, 30), (2000.0, 24), (0.0, 10)])
def test_lw_layer_count_matches_reference_formula(pkg, p_top, nk):
    from wrf_jax_b200 import _capi
    lib = _capi.load()
    # rrtmg_lw_nlayers (module_ra_rrtmg_common.py:1243-1247)
    expected = (nk + 1) + int(float(p_top) * 0.01 / 4.0 + 0.5) - 1
    assert lib.rrtmg_lw_nlayers(p_top, nk) == expected


def test_status_strings(pkg):
    from wrf_jax_b200 import _capi
    lib = _capi.load()
    assert lib.rrtmg_status_string(0) == b"ok"
    assert lib.rrtmg_status_string(2) == b"unsupported option"


def test_create_rejects_missing_blob(pkg):
    from wrf_jax_b200 import _capi
    lib = _capi.load()
    h = ctypes.c_void_p()
    st = lib.rrtmg_create(b"/nonexistent/blob.bin", 0, ctypes.byref(h))
    assert st == 1  # RRTMG_BAD_ARG, before any CUDA call
    assert b"cannot open" in lib.rrtmg_last_error(None)


def _one_entry_blob(dtype: int, ndim: int, shape, offset: int, nbytes: int, payload: bytes = b"") -> bytes:
    import struct
    head = b"RRTMGB2\0" + struct.pack("<II", 1, 1)
    entry = b"x".ljust(48, b"\0") + struct.pack("<II4IQQ", dtype, ndim, *shape, offset, nbytes)
    return head + entry + payload


@pytest.mark.parametrize("desc,blob", [
    # offset + nbytes wraps past 2**64: must not pass the range check
    ("wrapping range", _one_entry_blob(0, 1, (4, 1, 1, 1), 104, 2**64 - 8, b"\0" * 16)),
    # inside the buffer, but nbytes is not 4 * (3 x 2) floats
    ("size vs shape", _one_entry_blob(0, 2, (3, 2, 1, 1), 104, 16, b"\0" * 16)),
    ("unknown dtype", _one_entry_blob(7, 1, (4, 1, 1, 1), 104, 16, b"\0" * 16)),
])
def test_create_rejects_malformed_blob_before_any_cuda_call(pkg, desc, blob):
    """rrtmg_create_from_memory parses the blob on the host first; a malformed
    entry is RRTMG_BAD_ARG, never an out-of-range read."""
    from wrf_jax_b200 import _capi
    lib = _capi.load()
    h = ctypes.c_void_p()
    buf = ctypes.create_string_buffer(blob, len(blob))
    st = lib.rrtmg_create_from_memory(buf, len(blob), 0, ctypes.byref(h))
    assert st == 1, desc
    msg = lib.rrtmg_last_error(None)
    assert b"table entry" in msg, (desc, msg)
