"""Radiation prologue without a GPU: the oracle against the reference's golden
fixtures, the package's host-side scalars, the C-ABI's host helpers and the
ozone file reader."""

from __future__ import annotations

import ctypes
import sys

import numpy as np
import pytest

from conftest import GOLDEN, REPO


@pytest.fixture(scope="module")
def pro_golden():
    with np.load(GOLDEN / "prologue_golden.npz") as d:
        data = {k: d[k] for k in d.files}
    cases = {}
    for key, value in data.items():
        parts = key.split("/")
        if parts[0] == "ozone":
            cases.setdefault("ozone", {})[parts[1]] = value
        elif parts[1] == "in":
            cases.setdefault(parts[0], {}).setdefault("in", {})[parts[2]] = value
        else:
            cases.setdefault(parts[0], {})[parts[1]] = value
    return cases


@pytest.fixture(scope="module")
def po():
    sys.path.insert(0, str(REPO / "oracle"))
    import prologue_oracle
    return prologue_oracle


def _cases(g):
    return sorted(k for k in g if k != "ozone")


def _ulps(a, b):
    ia = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    ib = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(ia - ib)


def test_oracle_matches_reference_golden(pro_golden, po):
    g = pro_golden
    oz = g["ozone"]
    for name in _cases(g):
        c = g[name]
        i = c["in"]
        julian, xtime, gmt = (float(v) for v in i["calendar"])
        declin, solcon = po.radconst(julian)
        np.testing.assert_array_equal(np.float64([declin, solcon]), c["radconst"], err_msg=name)
        np.testing.assert_array_equal(np.float64(po.ozone_month_weights(julian)), c["month_weights"], err_msg=name)
        for gg in (0, 1, 2):
            np.testing.assert_array_equal(np.float32(po.greenhouse_scalars(2019, gg)), c[f"ghg{gg}"])
        cz = po.calc_coszen(i["xlat"], i["xlong"], julian=julian, xtime=xtime, gmt=gmt, declin=declin)
        np.testing.assert_array_equal(cz, c["coszen"], err_msg=f"{name} coszen")
        o3 = po.cam_o3rad(i["xlat"], i["p3d"], julian=julian, plev=oz["plev_pa"], lat_oz=oz["lat"],
                          ozone=oz["ozone"])
        np.testing.assert_array_equal(o3, c["o33d"], err_msg=f"{name} o33d")
        # numpy's float32 exp/power are the reference's; on another CPU their
        # SIMD variants may differ in the last place, nowhere near a threshold
        cf = po.cal_cldfra1(i["qv3d"], i["qc3d"], i["qi3d"], i["qs3d"], i["t3d"], i["p3d"])
        assert np.array_equal(cf == 0, c["cldfra"] == 0) and np.array_equal(cf == 1, c["cldfra"] == 1), name
        assert _ulps(cf, c["cldfra"]).max() <= 4, name


def test_golden_cases_cover_the_branches(pro_golden):
    g = pro_golden
    plev = g["ozone"]["plev_pa"]
    above = below = tails = wraps = 0
    for name in _cases(g):
        p = g[name]["in"]["p3d"]
        above += int(np.sum(p < plev[0]))
        below += int(np.sum(p > plev[-1]))
        tails += g[name]["in"]["xlat"].shape[0] % 4
        wraps += int(g[name]["month_weights"][1] == 0)
        cf = g[name]["cldfra"]
        assert np.any(cf == 1) and np.any((cf > 0) & (cf < 1)), name
    assert above and below and tails and wraps >= 2


def test_package_scalars_equal_reference(pkg, pro_golden):
    from wrf_jax_b200 import prologue
    for name in _cases(pro_golden):
        c = pro_golden[name]
        julian = float(c["in"]["calendar"][0])
        assert np.float64(prologue.radconst(julian)).tolist() == c["radconst"].tolist()
        assert np.float64(prologue.ozone_month_weights(julian)).tolist() == c["month_weights"].tolist()
        for gg in (0, 1, 2):
            np.testing.assert_array_equal(np.float32(prologue.greenhouse_scalars(2019, gg)), c[f"ghg{gg}"])


def test_package_coszen_scalars_equal_oracle(pkg, po, pro_golden):
    from wrf_jax_b200 import prologue
    for name in _cases(pro_golden):
        julian, xtime, gmt = (float(v) for v in pro_golden[name]["in"]["calendar"])
        declin = float(pro_golden[name]["radconst"][0])
        sc = prologue.prologue_scalars(julian=julian, xtime=xtime, gmt=gmt, declin=declin)
        assert (sc.tloctm0, sc.sin_declin, sc.cos_declin) == tuple(
            float(np.float32(v)) for v in po.coszen_scalars(julian, xtime, gmt, declin))
        lo, hi, w1, w2 = po.ozone_month_weights(julian)
        assert (sc.month_lo, sc.month_hi, sc.fact_lo, sc.fact_hi) == (lo, hi, np.float32(w1), np.float32(w2))


def test_c_abi_scalar_helpers(pkg, po):
    """The C helpers use the host libm for sin/cos/asin (numpy's float32 SIMD
    versions can differ in the last place); month weights are exact."""
    from wrf_jax_b200 import _capi
    lib = _capi.load()
    for julian in (0.0, 5.4, 15.0, 79.99, 80.0, 172.3, 355.2, 364.5, 365.9):
        d, s = ctypes.c_float(), ctypes.c_float()
        assert lib.rrtmg_radconst(julian, ctypes.byref(d), ctypes.byref(s)) == 0
        rd, rs = po.radconst(julian)
        assert _ulps(d.value, rd) <= 2 and _ulps(s.value, rs) <= 1
        sc = _capi.PrologueScalars()
        assert lib.rrtmg_prologue_scalars_from_calendar(julian, 1234.5, 6.0, rd, ctypes.byref(sc)) == 0
        t0, sd, cd = po.coszen_scalars(julian, 1234.5, 6.0, rd)
        assert _ulps(sc.tloctm0, t0) <= 2 and _ulps(sc.sin_declin, sd) <= 1 and _ulps(sc.cos_declin, cd) <= 1
        lo, hi, w1, w2 = po.ozone_month_weights(julian)
        assert (sc.month_lo, sc.month_hi) == (lo, hi)
        assert (np.float32(sc.fact_lo), np.float32(sc.fact_hi)) == (np.float32(w1), np.float32(w2))
    bad = _capi.PrologueScalars()
    assert lib.rrtmg_prologue_scalars_from_calendar(float("nan"), 0.0, 0.0, 0.0, ctypes.byref(bad)) == 1


def test_ozone_files_round_trip(pkg, tmp_path, pro_golden):
    from wrf_jax_b200 import prologue, synthetic
    plev_hpa, lat, oz = synthetic.cam_ozone_climatology(seed=0)
    synthetic.write_cam_ozone_files(tmp_path, plev_hpa, lat, oz)
    plev_pa, lat2, oz2 = prologue.load_cam_ozone_tables(tmp_path)
    np.testing.assert_array_equal(plev_pa, pro_golden["ozone"]["plev_pa"])
    np.testing.assert_array_equal(lat2, pro_golden["ozone"]["lat"])
    np.testing.assert_array_equal(oz2, pro_golden["ozone"]["ozone"])


def test_set_ozone_rejects_bad_climatology_without_gpu(pkg):
    """Argument checks run before any CUDA call."""
    from wrf_jax_b200 import _capi
    lib = _capi.load()
    plev = np.asarray([100.0, 50.0, 200.0], np.float32)  # not ascending
    lat = np.asarray([-10.0, 10.0], np.float32)
    oz = np.zeros((12, 2, 3), np.float32)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    assert lib.rrtmg_set_ozone_climatology(None, ptr(plev), 3, ptr(lat), 2, ptr(oz)) == 1
    assert lib.rrtmg_radiation_prologue(None, 1, 1, 1, None, None, None, None) == 1
