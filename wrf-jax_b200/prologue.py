"""Radiation prologue on B200: the per-step inputs of the RRTMG calls.

WRF-JAX's radiation stage derives three fields before it calls RRTMG
(``_radiation_driver_stage``, src/wrf_jax/runtime.py:7733-7766).  This module
computes them with librrtmg_b200.so (``include/rrtmg_prologue.h``), under the
reference's names and keywords:

* ``cal_cldfra1(qv, qc, qi, qs, t_phy, p_phy)``              runtime.py:5896 / 5967
* ``calc_coszen(xlat, xlong, *, julian, xtime, gmt, declin)`` runtime.py:6207 / 6246
* ``cam_o3rad(xlat, p3d, *, julian, case_dir)``               runtime.py:5804

and all of them in one launch, ``radiation_prologue``.  The per-step scalars
(``radconst``, the equation of time, the ozone month weights, the greenhouse
gases) stay host work as in the reference and are computed here with numpy in
the reference's binary32 statement order, so that they equal the reference's
host values bit for bit.

Arrays are float32 in the WRF runtime layout, numpy (copied to the GPU, results
copied back) or torch CUDA tensors (results stay on the GPU).  There is no CPU
path: without the library or a CUDA device the calls raise.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path
from typing import Any, NamedTuple

import numpy as np

from . import _capi
from .rrtmg import RrtmgContext, _as_device, _check_rounding_token, default_context

f32 = np.float32


# ---------------------------------------------------------------------------
# per-step scalars (host)
# ---------------------------------------------------------------------------
def radconst(julian: float) -> tuple[float, float]:
    """Declination [rad] and solar constant [W m-2] (runtime.py:5667-5690)."""
    degrad = f32(np.pi / 180.0)
    jr = f32(julian)
    dpd = f32(f32(360.0) / f32(365.0))
    sinob = f32(np.sin(f32(f32(23.5) * degrad)))
    days = f32(jr - f32(80.0)) if jr >= f32(80.0) else f32(jr + f32(285.0))
    sxlong = f32(f32(dpd * days) * degrad)
    declin = f32(np.arcsin(f32(sinob * f32(np.sin(sxlong)))))
    rjul = f32(f32(f32(jr * f32(360.0)) / f32(365.0)) * degrad)
    rjul2 = f32(f32(2.0) * rjul)
    ecc = f32(1.000110)
    for coef, fn, arg in ((0.034221, np.cos, rjul), (0.001280, np.sin, rjul),
                          (0.000719, np.cos, rjul2), (0.000077, np.sin, rjul2)):
        ecc = f32(ecc + f32(f32(coef) * f32(fn(arg))))
    return float(declin), float(f32(f32(1370.0) * ecc))


def greenhouse_scalars(yr: int, ghg_input: int = 1) -> tuple:
    """(co2, n2o, ch4, cfc11, cfc12) volume mixing ratios without a CAM gas
    table (runtime.py:5640-5664); the table reader (ghg_input=1 with a case
    directory) is not part of this path."""
    co2 = (280.0 + 90.0 * np.exp(0.02 * (int(yr) - 2000))) * 1.0e-6 if int(ghg_input) == 0 else 379.0e-6
    return tuple(f32(v) for v in (co2, 319.0e-9, 1774.0e-9, 0.251e-9, 0.538e-9))


_MID_MONTH = np.asarray([16, 45, 75, 105, 136, 166, 197, 228, 258, 289, 319, 350], np.float32)


def ozone_month_weights(julian: float) -> tuple[int, int, float, float]:
    """CAM ozone months bracketing the date (0-based) and their weights
    (runtime.py:5717-5750)."""
    t = f32(f32(julian) + f32(1.0))
    whole = int(t)
    frac = f32(t - f32(whole))
    whole = whole % 365 or 365
    t = f32(frac + f32(whole))
    later = np.flatnonzero(_MID_MONTH > t)
    hi = int(later[0]) if later.size else 0
    lo = hi - 1 if hi > 0 else 11
    d_lo, d_hi = _MID_MONTH[lo], _MID_MONTH[hi]
    if hi > 0:
        span = f32(d_hi - d_lo)
        return lo, hi, float(f32(f32(d_hi - t) / span)), float(f32(f32(t - d_lo) / span))
    year = f32(365.0)
    span = f32(f32(d_hi + year) - d_lo)
    if t > d_hi:
        return lo, hi, float(f32(f32(f32(d_hi + year) - t) / span)), float(f32(f32(t - d_lo) / span))
    return lo, hi, float(f32(f32(d_hi - t) / span)), float(f32(f32(f32(t + year) - d_lo) / span))


def prologue_scalars(*, julian: float, xtime: float, gmt: float, declin: float) -> "_capi.PrologueScalars":
    """rrtmg_prologue_scalars of a step: the equation-of-time offset
    (runtime.py:6220-6234), sin/cos of the declination and the ozone months."""
    da = f32(f32(f32(6.2831853071795862) * f32(f32(julian) - f32(1.0))) / f32(365.0))
    da2 = f32(f32(2.0) * da)
    eot = f32(0.000075)
    for coef, fn, arg in ((0.001868, np.cos, da), (-0.032077, np.sin, da),
                          (-0.014615, np.cos, da2), (-0.04089, np.sin, da2)):
        term = f32(f32(abs(coef)) * f32(fn(arg)))
        eot = f32(eot + term) if coef > 0 else f32(eot - term)
    eot = f32(eot * f32(229.18))
    xt24 = f32(f32(np.fmod(f32(xtime), f32(1440.0))) + eot)
    tloc = f32(f32(gmt) + f32(xt24 / f32(60.0)))
    lo, hi, w1, w2 = ozone_month_weights(julian)
    return _capi.PrologueScalars(tloctm0=float(tloc), sin_declin=float(f32(np.sin(f32(declin)))),
                                 cos_declin=float(f32(np.cos(f32(declin)))), month_lo=lo, month_hi=hi,
                                 fact_lo=w1, fact_hi=w2)


def load_cam_ozone_tables(case_dir) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(plev [Pa], lat [deg], ozone (12, latsiz, levsiz)) from a case directory's
    ozone_plev.formatted, ozone_lat.formatted and ozone.formatted
    (runtime.py:5697-5714)."""
    base = Path(case_dir) if case_dir is not None else Path.cwd()
    plev = np.loadtxt(base / "ozone_plev.formatted", dtype=np.float32) * f32(100.0)
    lat = np.loadtxt(base / "ozone_lat.formatted", dtype=np.float32)
    raw = np.loadtxt(base / "ozone.formatted", dtype=np.float32)
    expected = 12 * lat.shape[0] * plev.shape[0]
    if raw.size != expected:
        raise ValueError(f"ozone.formatted has {raw.size} values, expected {expected}")
    return plev, lat, raw.reshape(12, lat.shape[0], plev.shape[0])


# ---------------------------------------------------------------------------
# ozone climatology on the context
# ---------------------------------------------------------------------------
_ozone_lock = threading.Lock()
_ozone_loaded: dict = {}  # id(context) -> key of the climatology it holds


def set_ozone_climatology(plev_pa, lat, ozone, *, context: RrtmgContext | None = None, key=None) -> None:
    """Copy a CAM ozone climatology to the context's GPU (replaces the previous one)."""
    ctx = context or default_context()
    plev_pa = np.ascontiguousarray(plev_pa, np.float32)
    lat = np.ascontiguousarray(lat, np.float32)
    ozone = np.ascontiguousarray(ozone, np.float32)
    if ozone.shape != (12, lat.shape[0], plev_pa.shape[0]):
        raise ValueError(f"ozone must have shape (12, latsiz, levsiz), got {ozone.shape}")
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    ctx.check(ctx.lib.rrtmg_set_ozone_climatology(ctx.handle, ptr(plev_pa), plev_pa.shape[0], ptr(lat),
                                                  lat.shape[0], ptr(ozone)))
    with _ozone_lock:
        _ozone_loaded[id(ctx)] = key


def _ensure_ozone(ctx: RrtmgContext, case_dir) -> None:
    key = str(Path(case_dir if case_dir is not None else Path.cwd()).resolve())
    with _ozone_lock:
        if _ozone_loaded.get(id(ctx)) == key:
            return
    set_ozone_climatology(*load_cam_ozone_tables(case_dir), context=ctx, key=key)


# ---------------------------------------------------------------------------
# device calls
# ---------------------------------------------------------------------------
class RadiationPrologue(NamedTuple):
    cldfra3d: Any            # (nx, nk, ny), or None when icloud == 0
    o33d: Any                # (nx, nk, ny)
    coszr: Any               # (nx, ny), at the middle of the radiation interval
    condensate_present: Any  # device int32 scalar tensor (host int for host inputs)
    declin: float
    solcon: float
    gases: tuple             # (co2, n2o, ch4, cfc11, cfc12)


def _run(ctx, nx, nk, ny, scalars, d: dict, outs: dict, stream) -> None:
    import torch

    cin = _capi.PrologueIn(**{k: (d[k].data_ptr() if k in d else None) for k in _capi.PROLOGUE_IN_FIELDS})
    cout = _capi.PrologueOut(**{k: (outs[k].data_ptr() if outs.get(k) is not None else None)
                                for k in _capi.PROLOGUE_OUT_FIELDS})
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    sp = ctypes.byref(scalars) if scalars is not None else None
    ctx.check(ctx.lib.rrtmg_radiation_prologue(ctx.handle, nx, nk, ny, sp, ctypes.byref(cin), ctypes.byref(cout),
                                               ctypes.c_void_p(s)))


def _shape3(d, names):
    shape = tuple(d[names[0]].shape)
    if len(shape) != 3:
        raise ValueError(f"{names[0]} must be (nx, nk, ny), got {shape}")
    for k in names:
        if tuple(d[k].shape) != shape:
            raise ValueError(f"{k} must have shape {shape}, got {tuple(d[k].shape)}")
    return shape


def _host_result(host: bool, t):
    import torch

    if not host or t is None:
        return t
    torch.cuda.current_stream().synchronize()
    return t.cpu().numpy()


def cal_cldfra1(qv, qc, qi, qs, t_phy, p_phy, *, context: RrtmgContext | None = None, stream=None, out=None):
    """WRF cal_cldfra1 cloud fraction (runtime.py:5896-5964), (nx, nk, ny)."""
    import torch

    ctx = context or default_context()
    with torch.cuda.device(ctx.device):
        d, host = _as_device(dict(qv3d=qv, qc3d=qc, qi3d=qi, qs3d=qs, t3d=t_phy, p3d=p_phy), ctx.device)
        nx, nk, ny = _shape3(d, ("qv3d", "qc3d", "qi3d", "qs3d", "t3d", "p3d"))
        res = out if out is not None else torch.empty((nx, nk, ny), dtype=torch.float32, device=f"cuda:{ctx.device}")
        _run(ctx, nx, nk, ny, None, d, {"cldfra3d": res}, stream)
        return _host_result(host, res)


def calc_coszen(xlat, xlong, *, julian: float, xtime: float, gmt: float, declin: float,
                context: RrtmgContext | None = None, stream=None, out=None):
    """cos(solar zenith angle) on (nx, ny) (runtime.py:6207-6243)."""
    import torch

    ctx = context or default_context()
    with torch.cuda.device(ctx.device):
        d, host = _as_device(dict(xlat=xlat, xlong=xlong), ctx.device)
        nx, ny = d["xlat"].shape
        if tuple(d["xlong"].shape) != (nx, ny):
            raise ValueError("xlat and xlong must have the same (nx, ny) shape")
        res = out if out is not None else torch.empty((nx, ny), dtype=torch.float32, device=f"cuda:{ctx.device}")
        sc = prologue_scalars(julian=julian, xtime=xtime, gmt=gmt, declin=declin)
        _run(ctx, nx, 1, ny, sc, d, {"coszr": res}, stream)
        return _host_result(host, res)


def cam_o3rad(xlat, p3d, *, julian: float, case_dir=None, rounding_token=None, context: RrtmgContext | None = None,
              stream=None, out=None):
    """Ozone volume mixing ratio (nx, nk, ny) from the case's CAM climatology
    (runtime.py:5804-5819); the climatology is read once per case directory.
    Pass ``case_dir=False`` to use the one set by ``set_ozone_climatology``."""
    import torch

    _check_rounding_token(rounding_token)
    ctx = context or default_context()
    if case_dir is not False:
        _ensure_ozone(ctx, case_dir)
    with torch.cuda.device(ctx.device):
        d, host = _as_device(dict(xlat=xlat, p3d=p3d), ctx.device)
        nx, nk, ny = _shape3(d, ("p3d",))
        if tuple(d["xlat"].shape) != (nx, ny):
            raise ValueError("xlat must be (nx, ny) of p3d's (nx, nk, ny)")
        res = out if out is not None else torch.empty((nx, nk, ny), dtype=torch.float32, device=f"cuda:{ctx.device}")
        lo, hi, w1, w2 = ozone_month_weights(julian)
        sc = _capi.PrologueScalars(month_lo=lo, month_hi=hi, fact_lo=w1, fact_hi=w2)
        _run(ctx, nx, nk, ny, sc, d, {"o33d": res}, stream)
        return _host_result(host, res)


def radiation_prologue(*, qv, qc, qi, qs, t3d, p3d, xlat, xlong, julian: float, xtime: float, gmt: float,
                       yr: int, radt: float = 0.0, ghg_input: int = 1, case_dir=None, icloud: int = 1,
                       context: RrtmgContext | None = None, stream=None, out: dict | None = None
                       ) -> RadiationPrologue:
    """The radiation stage's prologue (runtime.py:7733-7766) in one launch:
    cloud fraction (when ``icloud`` is 1), CAM ozone, cos zenith at the middle
    of the radiation interval (xtime + radt / 2, runtime.py:7743), the
    condensate flag, and the host scalars.  ``case_dir=False`` uses the
    climatology set by ``set_ozone_climatology``.  ``out``: optional dict of
    preallocated CUDA tensors (cldfra3d, o33d, coszr, condensate_present)."""
    import torch

    ctx = context or default_context()
    if case_dir is not False:
        _ensure_ozone(ctx, case_dir)
    declin, solcon = radconst(julian)
    gases = greenhouse_scalars(yr, ghg_input)
    sc = prologue_scalars(julian=julian, xtime=float(xtime) + float(radt) * 0.5, gmt=gmt, declin=declin)
    with torch.cuda.device(ctx.device):
        d, host = _as_device(dict(qv3d=qv, qc3d=qc, qi3d=qi, qs3d=qs, t3d=t3d, p3d=p3d, xlat=xlat, xlong=xlong),
                             ctx.device)
        nx, nk, ny = _shape3(d, ("qv3d", "qc3d", "qi3d", "qs3d", "t3d", "p3d"))
        for k in ("xlat", "xlong"):
            if tuple(d[k].shape) != (nx, ny):
                raise ValueError(f"{k} must be (nx, ny) = {(nx, ny)}")
        dev = f"cuda:{ctx.device}"
        outs = dict(out) if out is not None else {
            "cldfra3d": torch.empty((nx, nk, ny), dtype=torch.float32, device=dev) if int(icloud) == 1 else None,
            "o33d": torch.empty((nx, nk, ny), dtype=torch.float32, device=dev),
            "coszr": torch.empty((nx, ny), dtype=torch.float32, device=dev),
            "condensate_present": torch.empty((), dtype=torch.int32, device=dev),
        }
        if int(icloud) != 1:
            outs["cldfra3d"] = None
        _run(ctx, nx, nk, ny, sc, d, outs, stream)
        flag = outs["condensate_present"]
        if host:
            flag = int(_host_result(True, flag)) if flag is not None else None
        return RadiationPrologue(cldfra3d=_host_result(host, outs["cldfra3d"]), o33d=_host_result(host, outs["o33d"]),
                                 coszr=_host_result(host, outs["coszr"]), condensate_present=flag,
                                 declin=declin, solcon=solcon, gases=gases)
