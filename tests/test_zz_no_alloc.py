"""rrtmg_lwrad_static_scratch (the LW call that allocates nothing) against
rrtmg_lwrad, both called through the C-ABI on the same device inputs.

Tolerance: bit-for-bit.  Both entry points launch the same McICA and LW kernels;
only the address of the McICA scratch differs, so any difference is a defect.
Collected last (file name) so it also runs after every other GPU test in the
same process; it needs no state from them.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATIC_MASK_WORDS = 8 << 20  # capacity of the static scratch, in 32-bit mask words


@pytest.fixture(scope="module")
def env(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import _capi, rrtmg
    ctx = rrtmg.RrtmgContext()
    yield ctx, _capi, torch
    torch.cuda.synchronize()
    ctx.close()


def _device_call(env, st, fn_name):
    ctx, _capi, torch = env
    kw = st.lw_kwargs()
    dev = f"cuda:{ctx.device}"
    d = {k: torch.from_numpy(np.ascontiguousarray(kw[k], dtype=np.float32)).to(dev) for k in _capi.LW_IN_FIELDS}
    nx, nk, ny = d["t3d"].shape
    cfg = _capi.Config(nx=nx, ny=ny, nk=nk, p_top=float(kw["p_top"]), co2vmr=kw["co2vmr"], n2ovmr=kw["n2ovmr"],
                       ch4vmr=kw["ch4vmr"], cfc11vmr=kw["cfc11vmr"], cfc12vmr=kw["cfc12vmr"], solcon=0.0,
                       has_reqc=int(kw["has_reqc"]), has_reqi=int(kw["has_reqi"]), has_reqs=int(kw["has_reqs"]),
                       icloud=int(kw["icloud"]), cldovrlp=int(kw["cldovrlp"]))
    outs = {k: torch.full((nx, nk, ny) if k.startswith("rthraten") else (nx, ny), float("nan"),
                          dtype=torch.float32, device=dev) for k in _capi.LW_OUT_FIELDS}
    cin = _capi.LwIn(**{k: d[k].data_ptr() for k in _capi.LW_IN_FIELDS})
    cout = _capi.LwOut(**{k: outs[k].data_ptr() for k in _capi.LW_OUT_FIELDS})
    stream = torch.cuda.current_stream().cuda_stream
    fn = getattr(ctx.lib, fn_name)
    st_code = fn(ctx.handle, ctypes.byref(cfg), ctypes.byref(cin), ctypes.byref(cout), ctypes.c_void_p(stream))
    assert st_code == 0, ctx.lib.rrtmg_last_error(ctx.handle).decode()
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in outs.items()}


def _assert_same(got: dict, ref: dict, tag: str) -> None:
    for name, value in ref.items():
        np.testing.assert_array_equal(got[name], value, err_msg=f"{tag} {name}")


@pytest.mark.parametrize("nx,ny,nk,seed,extra", [
    (48, 40, 50, 21, dict(fractional_clouds=True)),
    (31, 17, 44, 22, dict(p_top=1000.0, has_req=True, cloud_p=0.6)),
])
def test_static_scratch_matches_allocating_call_twice(env, pkg, nx, ny, nk, seed, extra):
    from wrf_jax_b200 import synthetic
    st = synthetic.make_columns(nx, ny, nk, seed=seed, **extra)
    ref = _device_call(env, st, "rrtmg_lwrad")
    first = _device_call(env, st, "rrtmg_lwrad_static_scratch")
    second = _device_call(env, st, "rrtmg_lwrad_static_scratch")
    _assert_same(first, ref, "first call")
    _assert_same(second, ref, "second call")


def test_static_scratch_alternating_layer_counts(env, pkg):
    """Calls with different model tops (so different LW layer counts) in turn:
    each selects its own slot of the jump table written at set-up, nothing is
    copied per call, and every call equals rrtmg_lwrad bit for bit."""
    from wrf_jax_b200 import synthetic
    a = synthetic.make_columns(20, 12, 50, seed=31, fractional_clouds=True)               # p_top 50 hPa: nlay 63
    b = synthetic.make_columns(20, 12, 50, seed=32, fractional_clouds=True, p_top=1000.0)  # nlay 53
    ctx = env[0]
    assert ctx.lib.rrtmg_lw_nlayers(float(a.lw_kwargs()["p_top"]), 50) != \
        ctx.lib.rrtmg_lw_nlayers(float(b.lw_kwargs()["p_top"]), 50)
    ref_a = _device_call(env, a, "rrtmg_lwrad")
    ref_b = _device_call(env, b, "rrtmg_lwrad")
    for rep in range(2):
        _assert_same(_device_call(env, a, "rrtmg_lwrad_static_scratch"), ref_a, f"round {rep} top 50 hPa")
        _assert_same(_device_call(env, b, "rrtmg_lwrad_static_scratch"), ref_b, f"round {rep} top 10 hPa")


def test_static_scratch_rejects_domain_beyond_capacity(env, pkg):
    ctx, _capi, torch = env
    nk, p_top = 50, 5000.0
    nlay = ctx.lib.rrtmg_lw_nlayers(p_top, nk)
    nx = 64
    ny = STATIC_MASK_WORDS // (nlay * 5 * nx) + 1  # one row of columns past the limit
    assert nlay * 5 * nx * ny > STATIC_MASK_WORDS
    dev = f"cuda:{ctx.device}"
    # real, correctly sized buffers: the call must refuse on the host before touching them
    three = torch.zeros((nx, nk, ny), dtype=torch.float32, device=dev)
    lev = torch.zeros((nx, nk + 1, ny), dtype=torch.float32, device=dev)
    two = torch.zeros((nx, ny), dtype=torch.float32, device=dev)
    levels = {"p8w", "t8w"}
    flat = {"tsk", "emiss", "xland", "xice", "snow"}
    cin = _capi.LwIn(**{k: (lev if k in levels else two if k in flat else three).data_ptr()
                        for k in _capi.LW_IN_FIELDS})
    cout = _capi.LwOut(**{k: (three if k.startswith("rthraten") else two).data_ptr() for k in _capi.LW_OUT_FIELDS})
    cfg = _capi.Config(nx=nx, ny=ny, nk=nk, p_top=p_top, co2vmr=4e-4, n2ovmr=3e-7, ch4vmr=1.7e-6, cfc11vmr=2e-10,
                       cfc12vmr=5e-10, solcon=0.0, has_reqc=0, has_reqi=0, has_reqs=0, icloud=1, cldovrlp=2)
    st_code = ctx.lib.rrtmg_lwrad_static_scratch(ctx.handle, ctypes.byref(cfg), ctypes.byref(cin),
                                                 ctypes.byref(cout), None)
    assert st_code == 1  # RRTMG_BAD_ARG
    assert b"static McICA scratch" in ctx.lib.rrtmg_last_error(ctx.handle)
