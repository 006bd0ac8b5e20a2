"""Radiation prologue on the GPU (through the C-ABI) against the reference's
golden fixtures and the CPU oracle.

Bars: ozone and cos zenith bit-exact (the same binary32 operations; SVML
emulation and glibc sinf/cosf restated).  Cloud fraction: the kernels call
CUDA expf/powf where the reference calls numpy's float32 exp and power (each
within a few units in the last place).  99.9 % of the values agree within
4e-7 absolute plus 2e-6 relative (1 - exp(arg) turns an exp difference of a
few ulp of 1 into that absolute error) and all within 2e-5 absolute: near
saturation the subsaturation qvs - qv cancels, and its power 0.49 carries the
saturation pressure's last-place difference into the exponent.  The 0 / 1
decisions agree except where the oracle's own value lies within 2e-5 of the
0.01 cut or 1e-4 of saturation.
"""

from __future__ import annotations

import sys

import numpy as np
import pytest

from conftest import GOLDEN, REPO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pro(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import prologue
    return prologue


@pytest.fixture(scope="module")
def po():
    sys.path.insert(0, str(REPO / "oracle"))
    import prologue_oracle
    return prologue_oracle


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLDEN / "prologue_golden.npz") as d:
        return {k: d[k] for k in d.files}


@pytest.fixture(scope="module")
def ozone_set(pro, gold):
    pro.set_ozone_climatology(gold["ozone/plev_pa"], gold["ozone/lat"], gold["ozone/ozone"], key="golden")
    return True


CASES = ("summer_7x5x44", "wrap_dec_4x6x50", "wrap_jan_9x3x30", "yearend_2x4x44", "spring_13x2x50")


def _ulps(a, b):
    ia = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    ib = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(ia - ib)


def assert_cldfra_close(got, want, inputs, po, tag=""):
    """Values as the module docstring states; decisions (0 / 1 / in between)
    equal except at borderline cases."""
    got = np.asarray(got, np.float32)
    want = np.asarray(want, np.float32)
    rhum, partial = po.cal_cldfra1_parts(*inputs)
    both = (got > 0) & (got < 1) & (want > 0) & (want < 1)
    diff = np.abs(got[both].astype(np.float64) - want[both])
    assert diff.max(initial=0.0) <= 2e-5, tag
    tight = diff <= 4e-7 + 2e-6 * np.abs(want[both])
    assert tight.sum() >= 0.999 * tight.size, f"{tag}: {int((~tight).sum())} of {tight.size} beyond 4e-7 + 2e-6 rel"
    differ = ((got == 0) != (want == 0)) | ((got == 1) != (want == 1))
    borderline = (np.abs(partial - np.float32(0.01)) <= 2e-5) | (np.abs(rhum - np.float32(1.0)) <= 1e-4)
    assert np.all(borderline[differ]), f"{tag}: {int(differ.sum())} decisions differ away from a threshold"
    assert differ.sum() <= max(2, got.size // 10000), tag


@pytest.mark.parametrize("case", CASES)
def test_prologue_matches_reference_golden(pro, po, gold, ozone_set, case):
    g = lambda k: gold[f"{case}/{k}"]
    julian, xtime, gmt = (float(v) for v in g("in/calendar"))
    r = pro.radiation_prologue(qv=g("in/qv3d"), qc=g("in/qc3d"), qi=g("in/qi3d"), qs=g("in/qs3d"),
                               t3d=g("in/t3d"), p3d=g("in/p3d"), xlat=g("in/xlat"), xlong=g("in/xlong"),
                               julian=julian, xtime=xtime, gmt=gmt, yr=2019, radt=0.0, case_dir=False)
    np.testing.assert_array_equal(r.coszr, g("coszen"), err_msg=f"{case} coszen")
    np.testing.assert_array_equal(r.o33d, g("o33d"), err_msg=f"{case} o33d")
    inputs = tuple(g(f"in/{k}") for k in ("qv3d", "qc3d", "qi3d", "qs3d", "t3d", "p3d"))
    assert_cldfra_close(r.cldfra3d, g("cldfra"), inputs, po, case)
    assert (r.declin, r.solcon) == tuple(g("radconst"))
    assert r.condensate_present == 1


def test_single_output_calls_equal_the_fused_call(pro, gold, ozone_set):
    import torch
    case = "summer_7x5x44"
    g = lambda k: torch.from_numpy(gold[f"{case}/{k}"]).cuda()
    julian, xtime, gmt = (float(v) for v in gold[f"{case}/in/calendar"])
    declin, _ = pro.radconst(julian)
    fused = pro.radiation_prologue(qv=g("in/qv3d"), qc=g("in/qc3d"), qi=g("in/qi3d"), qs=g("in/qs3d"),
                                   t3d=g("in/t3d"), p3d=g("in/p3d"), xlat=g("in/xlat"), xlong=g("in/xlong"),
                                   julian=julian, xtime=xtime, gmt=gmt, yr=2019, case_dir=False)
    cf = pro.cal_cldfra1(g("in/qv3d"), g("in/qc3d"), g("in/qi3d"), g("in/qs3d"), g("in/t3d"), g("in/p3d"))
    cz = pro.calc_coszen(g("in/xlat"), g("in/xlong"), julian=julian, xtime=xtime, gmt=gmt, declin=declin)
    oz = pro.cam_o3rad(g("in/xlat"), g("in/p3d"), julian=julian, case_dir=False)
    for a, b in ((cf, fused.cldfra3d), (cz, fused.coszr), (oz, fused.o33d)):
        assert torch.equal(a.view(torch.int32), b.view(torch.int32))
    assert int(fused.condensate_present.item()) == 1


@pytest.mark.parametrize("nx,ny,nk", [(262, 131, 50), (3, 4096, 44)])
def test_prologue_matches_oracle_large(pro, po, gold, ozone_set, nx, ny, nk):
    """Whole grids through the oracle: the SVML rows, the glibc tail rows (nx % 4)
    over a full range of latitudes, longitudes and hour angles, and the ozone
    and cloud branches."""
    from wrf_jax_b200 import synthetic
    st = synthetic.make_columns(nx=nx, ny=ny, nk=nk, seed=nx + ny)
    xlat, xlong = synthetic.lat_lon(nx, ny, seed=nx)
    f = {k: st.fields[k] for k in ("qv3d", "qc3d", "qi3d", "qs3d", "t3d", "p3d")}
    f["qv3d"] = (f["qv3d"] * np.float32(1.3)).astype(np.float32)
    for julian, xtime, gmt in ((172.3, 195.0, 6.0), (355.2, 2000.0, 23.5), (5.4, 0.0, 0.0)):
        declin, _ = po.radconst(julian)
        r = pro.radiation_prologue(qv=f["qv3d"], qc=f["qc3d"], qi=f["qi3d"], qs=f["qs3d"], t3d=f["t3d"],
                                   p3d=f["p3d"], xlat=xlat, xlong=xlong, julian=julian, xtime=xtime, gmt=gmt,
                                   yr=2019, case_dir=False)
        np.testing.assert_array_equal(
            r.coszr, po.calc_coszen(xlat, xlong, julian=julian, xtime=xtime, gmt=gmt, declin=declin))
        np.testing.assert_array_equal(
            r.o33d, po.cam_o3rad(xlat, f["p3d"], julian=julian, plev=gold["ozone/plev_pa"],
                                 lat_oz=gold["ozone/lat"], ozone=gold["ozone/ozone"]))
        inputs = tuple(f[k] for k in ("qv3d", "qc3d", "qi3d", "qs3d", "t3d", "p3d"))
        assert_cldfra_close(r.cldfra3d, po.cal_cldfra1(*inputs), inputs, po, f"{nx}x{ny}x{nk}")


def test_condensate_flag(pro):
    import torch
    nx, nk, ny = 5, 7, 33
    z = torch.zeros((nx, nk, ny), dtype=torch.float32, device="cuda")
    t = torch.full_like(z, 250.0)
    p = torch.full_like(z, 50000.0)

    def flag(qc, qi, qs):
        cf = torch.empty_like(z)
        r = torch.empty((), dtype=torch.int32, device="cuda")
        from wrf_jax_b200 import _capi
        import ctypes
        from wrf_jax_b200.rrtmg import default_context
        ctx = default_context()
        cin = _capi.PrologueIn(qv3d=z.data_ptr(), qc3d=qc.data_ptr(), qi3d=qi.data_ptr(), qs3d=qs.data_ptr(),
                               t3d=t.data_ptr(), p3d=p.data_ptr())
        cout = _capi.PrologueOut(cldfra3d=cf.data_ptr(), condensate_present=r.data_ptr())
        s = torch.cuda.current_stream().cuda_stream
        ctx.check(ctx.lib.rrtmg_radiation_prologue(ctx.handle, nx, nk, ny, None, ctypes.byref(cin),
                                                   ctypes.byref(cout), ctypes.c_void_p(s)))
        return int(r.item()), cf

    assert flag(z, z, z)[0] == 0
    neg0 = torch.full_like(z, -0.0)
    assert flag(neg0, neg0, z)[0] == 0                      # -0.0 has zero magnitude
    sub = z.clone()
    sub[4, 6, 32] = float(np.float32(1e-45))                # one subnormal anywhere sets it
    got, cf = flag(z, z, sub)
    assert got == 1 and float(cf.abs().max()) == 0.0        # but it is below the cloud minimum


def test_prologue_errors(pro):
    import torch
    from wrf_jax_b200.rrtmg import RrtmgError, RrtmgContext
    ctx = RrtmgContext()
    x = torch.zeros((4, 3), device="cuda")
    p = torch.full((4, 2, 3), 50000.0, device="cuda")
    with pytest.raises(RrtmgError, match="no ozone climatology"):
        pro.cam_o3rad(x, p, julian=10.0, case_dir=False, context=ctx)
    with pytest.raises(RrtmgError, match="ascending"):
        pro.set_ozone_climatology(np.asarray([3.0, 2.0, 1.0]), np.asarray([0.0, 1.0]), np.zeros((12, 2, 3)),
                                  context=ctx)
    with pytest.raises(ValueError):
        pro.cal_cldfra1(p, p, p, p, p, torch.zeros((4, 3), device="cuda"), context=ctx)
    ctx.close()
