"""XLA FFI handlers: the host-side checks, with this test playing XLA (no GPU
needed: every frame here is rejected before the handler touches the GPU)."""

from __future__ import annotations

import ctypes

import pytest

import xla_ffi_fake as X


@pytest.fixture(scope="module")
def lib(pkg):
    from wrf_jax_b200 import _capi
    return _capi.load()


def _lw_frame(xla, nx=3, nk=5, ny=4, drop_attr=None, bad_operand=None, ws_dtype=X.U8, n_operands=20):
    shapes = {"3": (nx, nk, ny), "L": (nx, nk + 1, ny), "2": (nx, ny)}
    kinds = "3L33L23333333" + "2222" + "333"
    ops = [(X.F32, 0x1000 + 256 * i, shapes[k]) for i, k in enumerate(kinds)][:n_operands]
    if bad_operand is not None:
        ops[bad_operand] = (X.F64, ops[bad_operand][1], ops[bad_operand][2])
    rets = [(X.F32, 0x9000 + 256 * i, shapes["3" if i < 2 else "2"]) for i in range(17)]
    rets.append((ws_dtype, 0x20000, (4096,)))
    attrs = {"p_top": (X.F64, 5000.0), "co2vmr": (X.F32, 4.1e-4), "n2ovmr": (X.F32, 3.19e-7),
             "ch4vmr": (X.F32, 1.774e-6), "cfc11vmr": (X.F32, 2.51e-10), "cfc12vmr": (X.F32, 5.38e-10),
             "has_reqc": (X.S32, 0), "has_reqi": (X.S32, 0), "has_reqs": (X.S32, 0), "icloud": (X.S32, 1),
             "cldovrlp": (X.S32, 2), "fp64_steps": (X.S32, 0)}
    if drop_attr:
        attrs.pop(drop_attr)
    return xla.frame(ops, rets, attrs)


def test_metadata_query(lib):
    xla = X.FakeXla()
    for name in ("rrtmg_ffi_lwrad", "rrtmg_ffi_swrad"):
        f, md = xla.metadata_frame()
        assert X.handler(lib, name)(ctypes.byref(f)) is None
        assert (md.api_version.major_version, md.api_version.minor_version, md.traits) == (0, 1, 0)
    assert not xla.errors


def test_stages_before_execute_do_nothing(lib):
    xla = X.FakeXla()
    for stage in (0, 1, 2):
        f = _lw_frame(xla)
        f.stage = stage
        assert X.handler(lib, "rrtmg_ffi_lwrad")(ctypes.byref(f)) is None
    assert not xla.errors


@pytest.mark.parametrize("kw,fragment", [
    (dict(n_operands=19), "takes 20 operands"),
    (dict(bad_operand=7), "operand 7"),
    (dict(drop_attr="p_top"), "missing attribute p_top"),
    (dict(drop_attr="fp64_steps"), "missing attribute fp64_steps"),
    (dict(ws_dtype=X.F32), "uint8 workspace"),
])
def test_malformed_calls_return_invalid_argument(lib, kw, fragment):
    xla = X.FakeXla()
    f = _lw_frame(xla, **kw)
    assert X.handler(lib, "rrtmg_ffi_lwrad")(ctypes.byref(f)) is not None
    assert len(xla.errors) == 1
    code, msg = xla.errors[0]
    assert code == X.INVALID_ARGUMENT and fragment in msg, msg


def test_host_pointers_are_rejected(lib):
    """Well-formed frame whose data pointers are not device memory."""
    xla = X.FakeXla()
    f = _lw_frame(xla)
    assert X.handler(lib, "rrtmg_ffi_lwrad")(ctypes.byref(f)) is not None
    assert xla.errors[0][0] == X.INVALID_ARGUMENT and "device memory" in xla.errors[0][1]
