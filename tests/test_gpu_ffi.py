"""The workspace entry points (rrtmg_lwrad_ws / rrtmg_swrad_ws) and the XLA
FFI handlers built on them, on the GPU: results equal rrtmg_lwrad /
rrtmg_swrad bit for bit.  The test plays XLA's side of the FFI call
(tests/xla_ffi_fake.py): operand and result buffers, scalar attributes, the
stream, and a uint8 workspace result sized by the workspace query."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import xla_ffi_fake as X

pytestmark = pytest.mark.gpu

SF8 = ("alswvisdir", "alswvisdif", "alswnirdir", "alswnirdif")


@pytest.fixture(scope="module")
def env(pkg, blob_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import _capi, rrtmg
    ctx = rrtmg.RrtmgContext()
    lib = ctx.lib
    lib.rrtmg_ffi_set_table_blob.restype = ctypes.c_int
    lib.rrtmg_ffi_set_table_blob.argtypes = [ctypes.c_char_p]
    assert lib.rrtmg_ffi_set_table_blob(str(blob_path).encode()) == 0
    for name in ("rrtmg_ffi_lw_workspace_bytes", "rrtmg_ffi_sw_workspace_bytes"):
        getattr(lib, name).restype = ctypes.c_size_t
        getattr(lib, name).argtypes = [ctypes.c_int, ctypes.POINTER(_capi.Config)]
    for name in ("rrtmg_lw_workspace_bytes", "rrtmg_sw_workspace_bytes"):
        getattr(lib, name).restype = ctypes.c_size_t
        getattr(lib, name).argtypes = [ctypes.c_void_p, ctypes.POINTER(_capi.Config)]
    lib.rrtmg_lwrad_ws.restype = ctypes.c_int
    lib.rrtmg_lwrad_ws.argtypes = [ctypes.c_void_p, ctypes.POINTER(_capi.Config), ctypes.POINTER(_capi.LwIn),
                                   ctypes.POINTER(_capi.LwOut), ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    lib.rrtmg_swrad_ws.restype = ctypes.c_int
    lib.rrtmg_swrad_ws.argtypes = [ctypes.c_void_p, ctypes.POINTER(_capi.Config), ctypes.POINTER(_capi.SwIn),
                                   ctypes.POINTER(_capi.SwOut), ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    yield ctx, _capi, rrtmg, torch
    torch.cuda.synchronize()
    ctx.close()


def _setup(env, st, side, sf8=False):
    ctx, _capi, rrtmg, torch = env
    kw = st.lw_kwargs() if side == "lw" else st.sw_kwargs()
    fields = _capi.LW_IN_FIELDS if side == "lw" else _capi.SW_IN_FIELDS + (SF8 if sf8 else ())
    dev = f"cuda:{ctx.device}"
    d = {k: torch.from_numpy(np.ascontiguousarray(kw[k] if k in kw else st.fields[k], dtype=np.float32)).to(dev)
         for k in fields}
    nx, nk, ny = d["t3d"].shape
    if side == "lw":
        cfg = rrtmg.lw_config(nx, ny, nk, p_top=kw["p_top"], yr=kw["yr"], co2vmr=kw["co2vmr"],
                              n2ovmr=kw["n2ovmr"], ch4vmr=kw["ch4vmr"], cfc11vmr=kw["cfc11vmr"],
                              cfc12vmr=kw["cfc12vmr"], has_reqc=kw["has_reqc"], has_reqi=kw["has_reqi"],
                              has_reqs=kw["has_reqs"])
        out_fields = _capi.LW_OUT_FIELDS
    else:
        cfg = rrtmg.sw_config(nx, ny, nk, solcon=kw["solcon"], yr=kw["yr"], co2vmr=kw["co2vmr"],
                              n2ovmr=kw["n2ovmr"], ch4vmr=kw["ch4vmr"], has_reqc=kw["has_reqc"],
                              has_reqi=kw["has_reqi"], has_reqs=kw["has_reqs"])
        out_fields = _capi.SW_OUT_FIELDS
    return d, cfg, out_fields, (nx, nk, ny)


def _outputs(env, out_fields, shape):
    torch = env[3]
    nx, nk, ny = shape
    return {k: torch.full((nx, nk, ny) if k.startswith("rthraten") else (nx, ny), float("nan"),
                          dtype=torch.float32, device=f"cuda:{env[0].device}") for k in out_fields}


def _reference(env, d, cfg, out_fields, shape, side):
    ctx, _capi, _, torch = env
    outs = _outputs(env, out_fields, shape)
    if side == "lw":
        cin = _capi.LwIn(**{k: d[k].data_ptr() for k in _capi.LW_IN_FIELDS})
        cout = _capi.LwOut(**{k: outs[k].data_ptr() for k in out_fields})
        fn = ctx.lib.rrtmg_lwrad
    else:
        cin = _capi.SwIn(**{k: v.data_ptr() for k, v in d.items()})
        cout = _capi.SwOut(**{k: outs[k].data_ptr() for k in out_fields})
        fn = ctx.lib.rrtmg_swrad
    s = torch.cuda.current_stream().cuda_stream
    ctx.check(fn(ctx.handle, ctypes.byref(cfg), ctypes.byref(cin), ctypes.byref(cout), ctypes.c_void_p(s)))
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in outs.items()}


def _assert_same(got, ref, tag):
    for k, v in ref.items():
        np.testing.assert_array_equal(got[k], v, err_msg=f"{tag} {k}")


@pytest.mark.parametrize("side", ["lw", "sw"])
def test_workspace_calls_match(env, pkg, side):
    from wrf_jax_b200 import synthetic
    ctx, _capi, _, torch = env
    st = synthetic.make_columns(40, 33, 50, seed=41, fractional_clouds=True)
    d, cfg, out_fields, shape = _setup(env, st, side)
    ref = _reference(env, d, cfg, out_fields, shape, side)
    nbytes = getattr(ctx.lib, f"rrtmg_{side}_workspace_bytes")(ctx.handle, ctypes.byref(cfg))
    assert nbytes > 0
    ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=f"cuda:{ctx.device}")
    base = (ws.data_ptr() + 255) // 256 * 256
    for rep in range(2):
        outs = _outputs(env, out_fields, shape)
        In, Out = (_capi.LwIn, _capi.LwOut) if side == "lw" else (_capi.SwIn, _capi.SwOut)
        cin = In(**{k: v.data_ptr() for k, v in d.items()})
        cout = Out(**{k: outs[k].data_ptr() for k in out_fields})
        fn = getattr(ctx.lib, f"rrtmg_{side}rad_ws")
        s = torch.cuda.current_stream().cuda_stream
        ctx.check(fn(ctx.handle, ctypes.byref(cfg), ctypes.byref(cin), ctypes.byref(cout), base, nbytes,
                     ctypes.c_void_p(s)))
        torch.cuda.synchronize()
        _assert_same({k: v.cpu().numpy() for k, v in outs.items()}, ref, f"{side} round {rep}")
    # one byte short: refused before any launch
    cin = In(**{k: v.data_ptr() for k, v in d.items()})
    assert fn(ctx.handle, ctypes.byref(cfg), ctypes.byref(cin), ctypes.byref(cout), base, nbytes - 1, None) == 1


def _ffi_call(env, d, cfg, out_fields, shape, side, ws_bytes):
    ctx, _capi, _, torch = env
    nx, nk, ny = shape
    xla = X.FakeXla(stream=torch.cuda.current_stream().cuda_stream)
    ops = [(X.F32, t.data_ptr(), tuple(t.shape)) for t in d.values()]
    outs = _outputs(env, out_fields, shape)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=f"cuda:{ctx.device}")
    assert ws.data_ptr() % 256 == 0
    rets = [(X.F32, outs[k].data_ptr(), tuple(outs[k].shape)) for k in out_fields] + [(X.U8, ws.data_ptr(),
                                                                                          (ws_bytes,))]
    flags = {k: (X.S32, getattr(cfg, k)) for k in ("has_reqc", "has_reqi", "has_reqs", "icloud", "cldovrlp",
                                                    "fp64_steps")}
    if side == "lw":
        attrs = {"p_top": (X.F64, cfg.p_top), **{k: (X.F32, getattr(cfg, k)) for k in
                                                   ("co2vmr", "n2ovmr", "ch4vmr", "cfc11vmr", "cfc12vmr")}}
    else:
        attrs = {"solcon": (X.F32, cfg.solcon), **{k: (X.F32, getattr(cfg, k)) for k in
                                                    ("co2vmr", "n2ovmr", "ch4vmr")}}
    f = xla.frame(ops, rets, {**attrs, **flags})
    err = X.handler(ctx.lib, f"rrtmg_ffi_{side}rad")(ctypes.byref(f))
    assert err is None, xla.errors
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in outs.items()}


@pytest.mark.parametrize("side,sf8", [("lw", False), ("sw", False), ("sw", True)])
def test_ffi_handler_matches_c_abi_call(env, pkg, side, sf8):
    from wrf_jax_b200 import synthetic
    ctx, _capi, _, torch = env
    st = synthetic.make_columns(24, 20, 50, seed=43, fractional_clouds=True, night_fraction=0.2)
    if sf8:
        rng = np.random.default_rng(5)
        st.fields["xland"] = np.where(rng.uniform(size=(24, 20)) < 0.5, 1.0, 2.0).astype(np.float32)
        for k in SF8:
            st.fields[k] = rng.uniform(0.03, 0.5, size=(24, 20)).astype(np.float32)
    d, cfg, out_fields, shape = _setup(env, st, side, sf8)
    ref = _reference(env, d, cfg, out_fields, shape, side)
    ws_bytes = getattr(ctx.lib, f"rrtmg_ffi_{side}_workspace_bytes")(ctx.device, ctypes.byref(cfg))
    assert ws_bytes > 0
    for rep in range(2):
        _assert_same(_ffi_call(env, d, cfg, out_fields, shape, side, ws_bytes), ref, f"ffi {side} round {rep}")
