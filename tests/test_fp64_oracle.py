"""The binary64 build of the oracle and the FP64 mode of the binary32 one.

The binary64 build (oracle/fp64.h) stands for an FP64 run of the reference
path; it cannot be pinned to the reference itself (the reference rounds every
operation to binary32), so these tests check its construction: it runs the
same algorithm (results close to the binary32 oracle's), samples the same
McICA subcolumns, and the FP64 mode of the binary32 oracle changes only the
two steps it names."""

from __future__ import annotations

import numpy as np
import pytest


@pytest.fixture(scope="module")
def o64(blob_path):
    import os
    import sys
    from conftest import REPO
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as oracle_mod
    return oracle_mod.Oracle(blob_path, nthreads=os.cpu_count(), binary64=True)


@pytest.fixture(scope="module")
def domain(pkg):
    from wrf_jax_b200 import synthetic
    return synthetic.make_columns(12, 9, 50, seed=7, fractional_clouds=True)


def _heating_kday(a, kw):
    return np.asarray(a, np.float64) * np.asarray(kw["pi3d"], np.float64) * 86400.0


def test_binary64_build_runs_the_same_algorithm(oracle, o64, domain):
    """binary32 results lie within the binary32 error of the binary64 run:
    heating within 0.1 K/day, fluxes within 0.5 W/m2 (measured on the 425 x 425
    x 50 domain: 0.03 K/day and 0.07 W/m2 at most)."""
    for side in ("lw", "sw"):
        kw = domain.lw_kwargs() if side == "lw" else domain.sw_kwargs()
        a = getattr(oracle, side + "rad")(**kw)
        b = getattr(o64, side + "rad")(**kw)
        for name, v in a.items():
            assert np.asarray(b[name]).dtype == np.float64
            if name.startswith("rthraten"):
                err = np.abs(_heating_kday(v, kw) - _heating_kday(b[name], kw)).max()
                assert err < 0.1, (side, name, err)
            else:
                err = np.abs(np.asarray(v, np.float64) - np.asarray(b[name])).max()
                assert err < 0.5, (side, name, err)


def test_binary64_build_samples_the_same_subcolumns(oracle, o64, domain):
    """The McICA stream and its cloud decisions stay binary32 in every build."""
    for side in ("lw", "sw"):
        kw = domain.lw_kwargs() if side == "lw" else domain.sw_kwargs()
        a = getattr(oracle, side + "rad")(diagnostics=True, **kw)["diag"]["cldfmc"]
        b = getattr(o64, side + "rad")(diagnostics=True, **kw)["diag"]["cldfmc"]
        np.testing.assert_array_equal(a, b)
        assert a.any()


def test_fp64_mode_changes_only_its_two_steps(oracle, domain):
    nk = domain.fields["t3d"].shape[1]
    top = nk - 5
    kw = domain.lw_kwargs()
    a, b = oracle.lwrad(**kw), oracle.lwrad(fp64_steps=1, **kw)
    for name, v in a.items():
        if name.startswith("rthraten"):
            np.testing.assert_array_equal(v[:, :top], b[name][:, :top], err_msg=name)
            assert np.abs(_heating_kday(v, kw) - _heating_kday(b[name], kw)).max() < 1e-3
        else:  # LW fluxes do not go through either step
            np.testing.assert_array_equal(v, b[name], err_msg=name)
    kw = domain.sw_kwargs()
    a, b = oracle.swrad(**kw), oracle.swrad(fp64_steps=1, **kw)
    night = np.asarray(kw["coszr"]) <= 0
    changed = False
    for name, v in a.items():
        assert np.all(np.asarray(b[name])[night] == 0) if v.ndim == 2 and name != "coszr" else True
        changed |= not np.array_equal(v, b[name])
    assert changed, "the FP64 reftra changed no SW output"
    # direct-beam fields do not go through reftra or the heating difference
    for name in ("swddir", "swddni", "swddirc", "swddnic", "swdnt", "swdntc"):
        np.testing.assert_array_equal(a[name], b[name], err_msg=name)


def test_error_table_fixture_is_consistent():
    """The committed FP64 error table (oracle/fp64_errors.py on the 425 x 425 x
    50 domain) covers every output of both modes."""
    import json
    from conftest import GOLDEN
    t = json.loads((GOLDEN / "fp64_errors_425x425x50.json").read_text())
    assert t["columns"] == 425 * 425
    for side, n in (("lw", 13), ("sw", 18)):
        for mode in ("binary32", "fp64_mode"):
            assert len(t[side][mode]) == n, (side, mode)
            for name, e in t[side][mode].items():
                assert 0.0 <= e["rms"] <= e["max"], (side, mode, name)
