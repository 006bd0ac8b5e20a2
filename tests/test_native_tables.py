"""Native reader of the reference's RRTMG data files (include/rrtmg_tables.h):
the absorption tables it builds from RRTMG_LW_DATA / RRTMG_SW_DATA are the
blob's tables byte for byte (those are pinned to checksums of the reference's
own compressed tables by test_oracle_golden.py), and malformed files are
rejected.  No GPU needed; the data files exist only where the WRF-JAX sources
are."""

from __future__ import annotations

import re

import numpy as np
import pytest

from conftest import REFERENCE_PHYSICS

DATA = REFERENCE_PHYSICS / "data" / "rrtmg"
ABSORPTION = re.compile(r"^(lw|sw)\d+\.")

pytestmark = pytest.mark.skipif(not (DATA / "RRTMG_LW_DATA").exists(),
                                reason="RRTMG data files of the reference are not on this machine")


def _lib():
    from wrf_jax_b200 import _capi
    return _capi.load()


def test_native_tables_equal_the_blob(pkg, blob_path, tmp_path):
    from wrf_jax_b200 import tables
    full = tables.read_blob(blob_path)
    base = {k: v for k, v in full.items() if not ABSORPTION.match(k)}
    assert len(base) < len(full)
    tables.write_blob(base, tmp_path / "base.bin")
    out = tmp_path / "native.bin"
    st = _lib().rrtmg_blob_with_wrf_data(str(tmp_path / "base.bin").encode(), str(DATA / "RRTMG_LW_DATA").encode(),
                                         str(DATA / "RRTMG_SW_DATA").encode(), str(out).encode())
    assert st == 0, _lib().rrtmg_last_error(None)
    native = tables.read_blob(out)
    assert sorted(native) == sorted(full)
    for name, want in full.items():
        got = native[name]
        assert got.dtype == want.dtype and got.shape == want.shape, name
        assert got.tobytes() == want.tobytes(), name
    # the whole file is the package writer's layout
    assert out.read_bytes() == blob_path.read_bytes()


def test_malformed_data_files_are_rejected(pkg, blob_path, tmp_path):
    raw = (DATA / "RRTMG_LW_DATA").read_bytes()
    n = int.from_bytes(raw[:4], "big")  # first record's length, repeated after its body
    cases = {
        "truncated": raw[: len(raw) // 2],
        "bad_marker": raw[: 4 + n] + (n + 4).to_bytes(4, "big") + raw[8 + n:],
        "short_record": (n - 4).to_bytes(4, "big") + raw[4: n] + (n - 4).to_bytes(4, "big") + raw[8 + n:],
        "trailing": raw + b"\x00" * 8,
    }
    lib = _lib()
    for name, data in cases.items():
        path = tmp_path / name
        path.write_bytes(data)
        st = lib.rrtmg_blob_with_wrf_data(str(blob_path).encode(), str(path).encode(),
                                          str(DATA / "RRTMG_SW_DATA").encode(), str(tmp_path / "o.bin").encode())
        assert st == 1, name
        assert lib.rrtmg_last_error(None), name
    st = lib.rrtmg_blob_with_wrf_data(str(blob_path).encode(), b"/nonexistent/RRTMG_LW_DATA",
                                      str(DATA / "RRTMG_SW_DATA").encode(), str(tmp_path / "o.bin").encode())
    assert st == 1 and b"cannot open" in lib.rrtmg_last_error(None)
