"""Drop-in replacements for WRF-JAX's RRTMG radiation calls, running on B200.

``rrtmg_lwrad_wrf_columns`` and ``rrtmg_swrad_wrf_columns`` take the same
keyword arguments as the reference's functions
(src/wrf_jax/physics/module_ra_rrtmg_lw.py:6789, module_ra_rrtmg_sw.py:2386) and
return named tuples with the same fields (RrtmgLwWrfColumnResult, lw:499;
RrtmgSwWrfColumnResult, sw:617).

Arrays may be numpy arrays (host; copied to the GPU and results copied back) or
torch CUDA tensors (used in place; results are torch CUDA tensors), float32 in
the WRF runtime layout (nx, nk, ny) / (nx, nk+1, ny) / (nx, ny).  The work runs
in librrtmg_b200.so on the current torch CUDA stream.  There is no CPU path: if
the library or a CUDA device is missing the call raises.

Unsupported reference options raise NotImplementedError like the reference
does (cldprmc liquid/ice options, lw:5750-5753, sw:1438-1441); the CAM
greenhouse-gas table reader (ghg_input=1 with a case directory) is not part of
this path, so such calls must pass the gas mixing ratios explicitly.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path
from typing import Any, NamedTuple

import numpy as np

from . import _capi, tables


class RrtmgLwWrfColumnResult(NamedTuple):
    rthratenlw: Any
    rthratenlwc: Any
    lwupt: Any
    lwuptc: Any
    lwuptcln: Any
    lwdnt: Any
    lwdntc: Any
    lwdntcln: Any
    lwupb: Any
    lwupbc: Any
    lwupbcln: Any
    lwdnb: Any
    lwdnbc: Any
    lwdnbcln: Any
    glw: Any
    olr: Any
    lwcf: Any


class RrtmgSwWrfColumnResult(NamedTuple):
    rthratensw: Any
    rthratenswc: Any
    swupt: Any
    swuptc: Any
    swuptcln: Any
    swdnt: Any
    swdntc: Any
    swdntcln: Any
    swupb: Any
    swupbc: Any
    swupbcln: Any
    swdnb: Any
    swdnbc: Any
    swdnbcln: Any
    swcf: Any
    gsw: Any
    swddir: Any
    swddni: Any
    swddif: Any
    swdownc: Any
    swddnic: Any
    swddirc: Any
    coszr: Any


class RrtmgError(RuntimeError):
    """A failed C-ABI call; ``status`` is the rrtmg_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_capi.STATUS.get(status, status)}: {message}")
        self.status = status


class RrtmgContext:
    """One library context: tables resident on one CUDA device."""

    def __init__(self, blob_path: str | Path | None = None, device: int | None = None):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("rrtmg_b200 needs a CUDA device; there is no CPU fallback")
        self.lib = _capi.load()
        self.device = torch.cuda.current_device() if device is None else int(device)
        path = Path(blob_path) if blob_path is not None else tables.DEFAULT_BLOB
        if not path.exists():
            raise FileNotFoundError(f"table blob {path} is missing (built by tables.ensure_blob)")
        handle = ctypes.c_void_p()
        st = self.lib.rrtmg_create(str(path).encode(), self.device, ctypes.byref(handle))
        if st != 0:
            raise RrtmgError(st, self.lib.rrtmg_last_error(None).decode())
        self.handle = handle

    @classmethod
    def from_wrf_data(cls, lw_data, sw_data, base_blob=None, device: int | None = None) -> "RrtmgContext":
        """A context whose absorption tables are read natively from the
        reference's RRTMG_LW_DATA / RRTMG_SW_DATA files (include/rrtmg_tables.h);
        the other tables come from ``base_blob`` (default: the package's blob)."""
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("rrtmg_b200 needs a CUDA device; there is no CPU fallback")
        self = cls.__new__(cls)
        self.lib = _capi.load()
        self.device = torch.cuda.current_device() if device is None else int(device)
        base = Path(base_blob) if base_blob is not None else tables.DEFAULT_BLOB
        handle = ctypes.c_void_p()
        st = self.lib.rrtmg_create_with_wrf_data(str(base).encode(), str(lw_data).encode(), str(sw_data).encode(),
                                                 self.device, ctypes.byref(handle))
        if st != 0:
            raise RrtmgError(st, self.lib.rrtmg_last_error(None).decode())
        self.handle = handle
        return self

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.rrtmg_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, st: int) -> None:
        if st != 0:
            msg = self.lib.rrtmg_last_error(self.handle).decode()
            if st == 2:
                raise NotImplementedError(msg)
            raise RrtmgError(st, msg)

    # per-column status bits of rrtmg_last_column_errors (include/rrtmg_b200.h)
    COL_NONFINITE_INPUT = 0x1
    COL_NONFINITE_OUTPUT = 0x2
    COL_PRESSURE_ORDER = 0x4
    COL_TEMPERATURE_RANGE = 0x8
    COL_FRACTION_RANGE = 0x10

    def column_status(self, enable: bool = True) -> None:
        """Record a per-column status bitmask after every LW / SW call on this
        context (one extra launch per call) until disabled."""
        self.check(self.lib.rrtmg_column_status_enable(self.handle, int(bool(enable))))

    def last_column_errors(self, side: str, nx: int, ny: int, stream=None):
        """Status words of the last recorded ``side`` ("lw" or "sw") call as an
        (nx, ny) int32 CUDA tensor (the uint32 bits of include/rrtmg_b200.h)."""
        import torch

        out = torch.empty((nx, ny), dtype=torch.int32, device=f"cuda:{self.device}")
        s = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        self.check(self.lib.rrtmg_last_column_errors(self.handle, 0 if side == "lw" else 1, out.data_ptr(),
                                                     nx * ny, ctypes.c_void_p(s)))
        return out


_default_ctx: dict = {}
_ctx_lock = threading.Lock()


def default_context(device: int | None = None) -> RrtmgContext:
    import torch

    dev = torch.cuda.current_device() if device is None else int(device)
    with _ctx_lock:
        if dev not in _default_ctx:
            _default_ctx[dev] = RrtmgContext(device=dev)
        return _default_ctx[dev]


def _greenhouse(yr, ghg_input, case_dir, co2vmr, n2ovmr, ch4vmr, cfc11vmr, cfc12vmr, lw: bool):
    """Gas scalars as the reference adapters choose them (lw:6610-6630, sw:2371-2383)."""
    given = (co2vmr, n2ovmr, ch4vmr) + ((cfc11vmr, cfc12vmr) if lw else ())
    if all(v is not None for v in given):
        return given + (() if lw else (0.0, 0.0))
    if lw and int(ghg_input) == 1 and case_dir is not None:
        raise NotImplementedError("CAM greenhouse-gas tables are not part of this path; pass the gas scalars")
    if int(ghg_input) == 0:
        co2 = (280.0 + 90.0 * np.exp(0.02 * (int(yr) - 2000))) * 1.0e-6
    else:
        co2 = 379.0e-6
    d = [co2, 319.0e-9, 1774.0e-9, 0.251e-9, 0.538e-9]
    if lw:  # the LW adapter ignores partially given scalars
        return tuple(d)
    vals = [v if v is not None else dv for v, dv in zip(given, d)]
    return tuple(vals) + (0.0, 0.0)


def lw_config(nx: int, ny: int, nk: int, *, p_top, yr, ghg_input=1, case_dir=None, co2vmr=None, n2ovmr=None,
              ch4vmr=None, cfc11vmr=None, cfc12vmr=None, icloud=1, has_reqc=1, has_reqi=1, has_reqs=1,
              cldovrlp=2, fp64_steps=False) -> "_capi.Config":
    """rrtmg_config of an LW call: the scalar keywords of rrtmg_lwrad_wrf_columns
    (``fp64_steps``: the FP64 mode of include/rrtmg_b200.h; no counterpart in
    the reference)."""
    co2, n2o, ch4, cfc11, cfc12 = _greenhouse(yr, ghg_input, case_dir, co2vmr, n2ovmr, ch4vmr,
                                              cfc11vmr, cfc12vmr, lw=True)
    return _capi.Config(nx=nx, ny=ny, nk=nk, p_top=float(p_top), co2vmr=co2, n2ovmr=n2o, ch4vmr=ch4,
                        cfc11vmr=cfc11, cfc12vmr=cfc12, solcon=0.0, has_reqc=int(has_reqc),
                        has_reqi=int(has_reqi), has_reqs=int(has_reqs), icloud=int(icloud),
                        cldovrlp=int(cldovrlp), fp64_steps=int(bool(fp64_steps)))


def sw_config(nx: int, ny: int, nk: int, *, solcon, yr, ghg_input=1, co2vmr=None, n2ovmr=None, ch4vmr=None,
              icloud=1, has_reqc=1, has_reqi=1, has_reqs=1, cldovrlp=2, fp64_steps=False) -> "_capi.Config":
    """rrtmg_config of an SW call: the scalar keywords of rrtmg_swrad_wrf_columns
    (``fp64_steps`` as for lw_config)."""
    co2, n2o, ch4, _, _ = _greenhouse(yr, ghg_input, None, co2vmr, n2ovmr, ch4vmr, None, None, lw=False)
    return _capi.Config(nx=nx, ny=ny, nk=nk, p_top=0.0, co2vmr=co2, n2ovmr=n2o, ch4vmr=ch4, cfc11vmr=0.0,
                        cfc12vmr=0.0, solcon=float(np.float32(solcon)), has_reqc=int(has_reqc),
                        has_reqi=int(has_reqi), has_reqs=int(has_reqs), icloud=int(icloud),
                        cldovrlp=int(cldovrlp), fp64_steps=int(bool(fp64_steps)))


def _as_device(arrays: dict, device: int):
    """numpy or host torch tensors -> torch CUDA float32 (contiguous); torch CUDA
    tensors pass through.  Returns the tensors and whether any input was on the host."""
    import torch

    out = {}
    host = False
    for k, v in arrays.items():
        if isinstance(v, torch.Tensor) and not v.is_cuda:
            # host tensor (pinned memory copies asynchronously); results come back to the host
            host = True
            t = v.contiguous().float().to(device=f"cuda:{device}", non_blocking=v.is_pinned())
        elif isinstance(v, torch.Tensor):
            t = v.contiguous()
            if t.dtype != torch.float32:
                t = t.float()
        else:
            host = True
            t = torch.from_numpy(np.ascontiguousarray(np.asarray(v, dtype=np.float32))).to(
                device=f"cuda:{device}", non_blocking=False)
        out[k] = t
    return out, host


def _check_shapes(d: dict, nx: int, nk: int, ny: int, three: tuple, lev: tuple, two: tuple) -> None:
    for k in three:
        if tuple(d[k].shape) != (nx, nk, ny):
            raise ValueError(f"{k} must have shape (nx, nk, ny) = {(nx, nk, ny)}, got {tuple(d[k].shape)}")
    for k in lev:
        if tuple(d[k].shape) != (nx, nk + 1, ny):
            raise ValueError(f"{k} must have shape (nx, nk+1, ny) = {(nx, nk + 1, ny)}, got {tuple(d[k].shape)}")
    for k in two:
        if tuple(d[k].shape) != (nx, ny):
            raise ValueError(f"{k} must have shape (nx, ny) = {(nx, ny)}, got {tuple(d[k].shape)}")


def _check_rounding_token(token) -> None:
    """The runtime passes a uint32 token that is XORed into every binary32
    store (core/real_arithmetic.py:12-14, runtime.py:16329 sets it to 0).  A
    zero token is a plain REAL store, which is what the kernels do; nonzero
    tokens are diagnostic bit edits and are not supported."""
    if token is None:
        return
    if hasattr(token, "detach"):  # torch tensor
        token = token.detach().cpu().numpy()
    if np.any(np.asarray(token).astype(np.uint64) != 0):
        raise NotImplementedError("nonzero (diagnostic) rounding tokens are not supported")


def _check_outputs(out: dict, names, nx: int, nk: int, ny: int) -> None:
    import torch
    for k in names:
        t = out[k]
        shape = (nx, nk, ny) if k.startswith("rthraten") else (nx, ny)
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
                and tuple(t.shape) == shape):
            raise ValueError(f"out[{k!r}] must be a contiguous float32 CUDA tensor of shape {shape}")


def rrtmg_lwrad_wrf_columns(*, p3d, p8w, pi3d, t3d, t8w, tsk, dz8w, qv3d, qc3d, qi3d, qs3d, cldfra3d, o33d,
                            emiss, xland, xice, snow, re_cloud, re_ice, re_snow, p_top, yr, julian,
                            ghg_input=1, case_dir=None, cldovrlp=2, idcor=0, icloud=1, has_reqc=1,
                            has_reqi=1, has_reqs=1, co2vmr=None, n2ovmr=None, ch4vmr=None, cfc11vmr=None,
                            cfc12vmr=None, lookup_tables=None, spectral=None, pade_tables=None,
                            cloud_tables=None, setcoef_tables=None, rounding_token=None,
                            context: RrtmgContext | None = None, stream=None, out=None,
                            fp64_steps: bool = False) -> RrtmgLwWrfColumnResult:
    """B200 ``RRTMG_LWRAD`` (module_ra_rrtmg_lw.py:6789).  Table keywords are
    accepted for signature parity and ignored (the context owns the tables).
    ``out``: optional dict of preallocated float32 CUDA tensors, one per result
    field, written in place (used for CUDA-graph capture).  ``fp64_steps``:
    heating rates of the five highest model layers formed in binary64 (the
    FP64 mode; off by default, which reproduces the reference bit for bit)."""
    import torch

    del idcor, julian, lookup_tables, spectral, pade_tables, cloud_tables, setcoef_tables
    _check_rounding_token(rounding_token)
    ctx = context or default_context()
    arrays = dict(p3d=p3d, p8w=p8w, pi3d=pi3d, t3d=t3d, t8w=t8w, tsk=tsk, dz8w=dz8w, qv3d=qv3d, qc3d=qc3d,
                  qi3d=qi3d, qs3d=qs3d, cldfra3d=cldfra3d, o33d=o33d, emiss=emiss, xland=xland, xice=xice,
                  snow=snow, re_cloud=re_cloud, re_ice=re_ice, re_snow=re_snow)
    with torch.cuda.device(ctx.device):
        d, host = _as_device(arrays, ctx.device)
        nx, nk, ny = d["t3d"].shape
        _check_shapes(d, nx, nk, ny,
                      ("p3d", "pi3d", "t3d", "dz8w", "qv3d", "qc3d", "qi3d", "qs3d", "cldfra3d", "o33d",
                       "re_cloud", "re_ice", "re_snow"), ("p8w", "t8w"),
                      ("tsk", "emiss", "xland", "xice", "snow"))
        cfg = lw_config(nx, ny, nk, p_top=p_top, yr=yr, ghg_input=ghg_input, case_dir=case_dir, co2vmr=co2vmr,
                        n2ovmr=n2ovmr, ch4vmr=ch4vmr, cfc11vmr=cfc11vmr, cfc12vmr=cfc12vmr, icloud=icloud,
                        has_reqc=has_reqc, has_reqi=has_reqi, has_reqs=has_reqs, cldovrlp=cldovrlp,
                        fp64_steps=fp64_steps)
        outs = out if out is not None else {
            k: torch.empty((nx, nk, ny) if k.startswith("rthraten") else (nx, ny), dtype=torch.float32,
                           device=f"cuda:{ctx.device}") for k in _capi.LW_OUT_FIELDS}
        if out is not None:
            _check_outputs(out, _capi.LW_OUT_FIELDS, nx, nk, ny)
        cin = _capi.LwIn(**{k: d[k].data_ptr() for k in _capi.LW_IN_FIELDS})
        cout = _capi.LwOut(**{k: outs[k].data_ptr() for k in _capi.LW_OUT_FIELDS})
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        ctx.check(ctx.lib.rrtmg_lwrad(ctx.handle, ctypes.byref(cfg), ctypes.byref(cin), ctypes.byref(cout),
                                      ctypes.c_void_p(s)))
        if host:
            torch.cuda.current_stream().synchronize()
            return RrtmgLwWrfColumnResult(**{k: outs[k].cpu().numpy() for k in _capi.LW_OUT_FIELDS})
        return RrtmgLwWrfColumnResult(**outs)


def rrtmg_swrad_wrf_columns(*, p3d, p8w, pi3d, t3d, t8w, tsk, dz8w, qv3d, qc3d, qi3d, qs3d, cldfra3d, o33d,
                            albedo, coszr, xland, xice, snow, re_cloud, re_ice, re_snow, solcon, yr, julian,
                            ghg_input=1, cldovrlp=2, idcor=0, icloud=1, has_reqc=1, has_reqi=1, has_reqs=1,
                            sf_surface_physics=2, alswvisdir=None, alswvisdif=None, alswnirdir=None,
                            alswnirdif=None, co2vmr=None, n2ovmr=None, ch4vmr=None, lookup_tables=None,
                            spectral=None, pade_tables=None, cloud_tables=None, rounding_token=None,
                            context: RrtmgContext | None = None, stream=None, out=None,
                            fp64_steps: bool = False) -> RrtmgSwWrfColumnResult:
    """B200 ``rrtmg_swrad`` (module_ra_rrtmg_sw.py:2386); ``out`` as for the LW
    call.  ``fp64_steps``: the FP64 mode (reftra of nearly conservative layers
    and the top layers' heating rates in binary64; off by default)."""
    import torch

    del idcor, julian, lookup_tables, spectral, pade_tables, cloud_tables
    _check_rounding_token(rounding_token)
    # Noah-MP albedos only when the reference uses them (sw:2521)
    sf8 = int(sf_surface_physics) == 8 and all(v is not None for v in (alswvisdir, alswvisdif, alswnirdir,
                                                                        alswnirdif))
    ctx = context or default_context()
    arrays = dict(p3d=p3d, p8w=p8w, pi3d=pi3d, t3d=t3d, t8w=t8w, tsk=tsk, dz8w=dz8w, qv3d=qv3d, qc3d=qc3d,
                  qi3d=qi3d, qs3d=qs3d, cldfra3d=cldfra3d, o33d=o33d, albedo=albedo, coszr=coszr,
                  xland=xland, xice=xice, snow=snow, re_cloud=re_cloud, re_ice=re_ice, re_snow=re_snow)
    if sf8:
        arrays.update(alswvisdir=alswvisdir, alswvisdif=alswvisdif, alswnirdir=alswnirdir, alswnirdif=alswnirdif)
    with torch.cuda.device(ctx.device):
        d, host = _as_device(arrays, ctx.device)
        nx, nk, ny = d["t3d"].shape
        _check_shapes(d, nx, nk, ny,
                      ("p3d", "pi3d", "t3d", "dz8w", "qv3d", "qc3d", "qi3d", "qs3d", "cldfra3d", "o33d",
                       "re_cloud", "re_ice", "re_snow"), ("p8w", "t8w"),
                      ("tsk", "albedo", "coszr", "xland", "xice", "snow")
                      + (_capi.SW_ALBEDO_FIELDS if sf8 else ()))
        cfg = sw_config(nx, ny, nk, solcon=solcon, yr=yr, ghg_input=ghg_input, co2vmr=co2vmr, n2ovmr=n2ovmr,
                        ch4vmr=ch4vmr, icloud=icloud, has_reqc=has_reqc, has_reqi=has_reqi, has_reqs=has_reqs,
                        cldovrlp=cldovrlp, fp64_steps=fp64_steps)
        outs = out if out is not None else {
            k: torch.empty((nx, nk, ny) if k.startswith("rthraten") else (nx, ny), dtype=torch.float32,
                           device=f"cuda:{ctx.device}") for k in _capi.SW_OUT_FIELDS}
        if out is not None:
            _check_outputs(out, _capi.SW_OUT_FIELDS, nx, nk, ny)
        cin = _capi.SwIn(**{k: d[k].data_ptr() for k in _capi.SW_IN_FIELDS + (_capi.SW_ALBEDO_FIELDS if sf8 else ())})
        cout = _capi.SwOut(**{k: outs[k].data_ptr() for k in _capi.SW_OUT_FIELDS})
        s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
        ctx.check(ctx.lib.rrtmg_swrad(ctx.handle, ctypes.byref(cfg), ctypes.byref(cin), ctypes.byref(cout),
                                      ctypes.c_void_p(s)))
        if host:
            torch.cuda.current_stream().synchronize()
            return RrtmgSwWrfColumnResult(**{k: outs[k].cpu().numpy() for k in _capi.SW_OUT_FIELDS})
        return RrtmgSwWrfColumnResult(**outs)
