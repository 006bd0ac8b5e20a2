"""Pin the CPU oracle to the reference: golden fixtures produced by WRF-JAX's own
RRTMG code (tests/golden/make_golden.py) must be reproduced bit for bit."""

from __future__ import annotations

import hashlib
import json

import numpy as np
import pytest

from conftest import GOLDEN, case_kwargs

CASES = ("c0_4x4x44", "c1_3x5x50", "req_3x3x44", "fraccloud_ptop10_3x3x30", "allnight_2x3x44",
         "clearsky_allday_3x2x44", "overcast_2x2x40", "icloud0_2x2x44", "odd_1x3x17", "sf8_3x4x44")


@pytest.mark.parametrize("case", CASES)
def test_lw_oracle_matches_reference_bitwise(oracle, golden, case):
    got = oracle.lwrad(**case_kwargs(golden[case], "lw"))
    for name, ref in golden[case]["lw"].items():
        np.testing.assert_array_equal(np.asarray(got[name], np.float32), ref, err_msg=f"{case} lw {name}")


@pytest.mark.parametrize("case", CASES)
def test_sw_oracle_matches_reference_bitwise(oracle, golden, case):
    got = oracle.swrad(**case_kwargs(golden[case], "sw"))
    for name, ref in golden[case]["sw"].items():
        np.testing.assert_array_equal(np.asarray(got[name], np.float32), ref, err_msg=f"{case} sw {name}")


def test_table_blob_matches_reference_compression(blob_path, pkg):
    from wrf_jax_b200 import tables
    blob = tables.read_blob(blob_path)
    expected = json.loads((GOLDEN / "tables_sha256.json").read_text())
    assert expected
    for name, digest in expected.items():
        arr = np.ascontiguousarray(blob[name])
        assert hashlib.sha256(arr.tobytes()).hexdigest() == digest, name


def test_kiss_stream_matches_reference():
    """The oracle's sequential KISS equals the reference's jump-ahead stream."""
    import ctypes
    import sys
    from conftest import REPO
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as oracle_mod
    lib = ctypes.CDLL(str(oracle_mod.build()))
    lib.ora_kiss_step.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_float)]
    with np.load(GOLDEN / "kiss_golden.npz") as d:
        seeds, first5 = d["seeds"], d["first5"]
        streams = {150: d["skip150"], 1: d["skip1"]}
    for skip, ref in streams.items():
        for c in range(seeds.shape[0]):
            s = (ctypes.c_uint32 * 4)(*[int(np.uint32(v)) for v in seeds[c]])
            r = ctypes.c_float()
            for _ in range(skip):
                lib.ora_kiss_step(s, ctypes.byref(r))
            draws = []
            for _ in range(ref.shape[0]):
                lib.ora_kiss_step(s, ctypes.byref(r))
                draws.append(r.value)
            np.testing.assert_array_equal(np.asarray(draws, np.float32), ref[:, c])
    for c in range(seeds.shape[0]):
        s = (ctypes.c_uint32 * 4)(*[int(np.uint32(v)) for v in seeds[c]])
        r = ctypes.c_float()
        got = []
        for _ in range(5):
            lib.ora_kiss_step(s, ctypes.byref(r))
            got.append(r.value)
        np.testing.assert_array_equal(np.asarray(got, np.float32), first5[:, c])
