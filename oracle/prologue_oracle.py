"""CPU oracle of the radiation prologue (test infrastructure only).

A numpy restatement of the per-step inputs WRF-JAX's radiation stage derives
before the RRTMG calls (``_radiation_driver_stage``, src/wrf_jax/runtime.py:7700-7766):

* ``cal_cldfra1``     cloud fraction from humidity and condensate
                      (``_cal_cldfra1_np``, runtime.py:5896-5964);
* ``calc_coszen``     cosine of the solar zenith angle, with the four-lane
                      SVML sin/cos emulation for whole groups of four
                      west-east rows and host libm for the rest
                      (``_calc_coszen_np``, runtime.py:6207-6243; SVML kernels
                      runtime.py:6027-6096; libm tail runtime.py:6099-6119);
* ``cam_o3rad``       CAM ozone climatology interpolated in latitude, month
                      and pressure (``_cam_o3rad_np``, runtime.py:5753-5801;
                      month weights ``_cam_ozone_month_weights``, 5717-5750);
* ``radconst``        declination and solar constant (runtime.py:5667-5690);
* ``greenhouse_scalars`` CO2/N2O/CH4/CFC defaults (runtime.py:5627-5664).

Every statement is the reference's: the same binary32 operation, in the same
order, through the same numpy functions (so ``np.exp`` / ``**`` / ``np.sin``
round exactly as the reference's own numpy path does on the machine it runs
on).  Only tests use this module, as the checker.
"""

from __future__ import annotations

import ctypes
import ctypes.util

import numpy as np

f32 = np.float32


def _bits32(v: int) -> np.float32:
    return np.asarray(v, dtype=np.uint32).view(np.float32)[()]


# ---------------------------------------------------------------------------
# calendar scalars
# ---------------------------------------------------------------------------
def radconst(julian: float) -> tuple[float, float]:
    """(declination [rad], solar constant [W m-2]) as runtime.py:5667-5690 rounds them."""
    degrad = f32(np.pi / 180.0)
    dpd = f32(f32(360.0) / f32(365.0))
    jr = f32(julian)
    obecl = f32(f32(23.5) * degrad)
    sinob = f32(np.sin(obecl))
    if jr >= f32(80.0):
        sxlong = f32(dpd * f32(jr - f32(80.0)))
    else:
        sxlong = f32(dpd * f32(jr + f32(285.0)))
    sxlong = f32(sxlong * degrad)
    declin = f32(np.arcsin(f32(sinob * f32(np.sin(sxlong)))))
    djul = f32(f32(jr * f32(360.0)) / f32(365.0))
    rjul = f32(djul * degrad)
    twice = f32(f32(2.0) * rjul)
    ecc = f32(1.000110)
    ecc = f32(ecc + f32(f32(0.034221) * f32(np.cos(rjul))))
    ecc = f32(ecc + f32(f32(0.001280) * f32(np.sin(rjul))))
    ecc = f32(ecc + f32(f32(0.000719) * f32(np.cos(twice))))
    ecc = f32(ecc + f32(f32(0.000077) * f32(np.sin(twice))))
    return float(declin), float(f32(f32(1370.0) * ecc))


def greenhouse_scalars(yr: int, ghg_input: int) -> tuple:
    """Gas volume mixing ratios without a CAM gas table (runtime.py:5640-5664)."""
    if int(ghg_input) == 0:
        co2 = (280.0 + 90.0 * np.exp(0.02 * (int(yr) - 2000))) * 1.0e-6
    else:
        co2 = 379.0e-6
    return (f32(co2), f32(319.0e-9), f32(1774.0e-9), f32(0.251e-9), f32(0.538e-9))


_OZONE_MID_MONTH_DAYS = np.asarray([16, 45, 75, 105, 136, 166, 197, 228, 258, 289, 319, 350], np.float32)


def ozone_month_weights(julian: float) -> tuple[int, int, float, float]:
    """(previous month, next month, their weights) of the CAM ozone cycle (runtime.py:5717-5750)."""
    days = _OZONE_MID_MONTH_DAYS
    t = f32(f32(julian) + f32(1.0))
    whole = int(t)
    frac = f32(t - f32(whole))
    whole %= 365
    if whole == 0:
        whole = 365
    t = f32(frac + f32(whole))
    later = np.nonzero(days > t)[0]
    nxt = int(later[0]) if later.size else 0
    if nxt > 0:
        prv = nxt - 1
        span = f32(days[nxt] - days[prv])
        w1 = f32(f32(days[nxt] - t) / span)
        w2 = f32(f32(t - days[prv]) / span)
    else:
        prv = 11
        span = f32(f32(days[0] + f32(365.0)) - days[prv])
        if t > days[0]:
            w1 = f32(f32(f32(days[0] + f32(365.0)) - t) / span)
            w2 = f32(f32(t - days[prv]) / span)
        else:
            w1 = f32(f32(days[0] - t) / span)
            w2 = f32(f32(f32(t + f32(365.0)) - days[prv]) / span)
    return prv, nxt, float(w1), float(w2)


# ---------------------------------------------------------------------------
# cloud fraction
# ---------------------------------------------------------------------------
def cal_cldfra1(qv, qc, qi, qs, t, p) -> np.ndarray:
    """WRF cal_cldfra1 on float32 arrays (runtime.py:5896-5964), element by element."""
    qv, qc, qi, qs, t, p = (np.asarray(a, np.float32) for a in (qv, qc, qi, qs, t, p))
    alpha0, gamma, qcldmin, pexp, rhgrid = f32(100.0), f32(0.49), f32(1.0e-12), f32(0.25), f32(1.0)
    svp1, svp2, svpi2, svp3, svpi3, svpt0 = (f32(0.61078), f32(17.2693882), f32(21.8745584),
                                             f32(35.86), f32(7.66), f32(273.15))
    ep_2 = f32(287.0 / 461.6)
    valid = (t > f32(100.0)) & (p > f32(100.0))
    ts = np.where(valid, t, svpt0)
    tc = ts - svpt0
    esw = f32(1000.0) * svp1 * np.exp(svp2 * tc / (ts - svp3)).astype(np.float32)
    esi = f32(1000.0) * svp1 * np.exp(svpi2 * tc / (ts - svpi3)).astype(np.float32)
    esw = np.where(valid, esw, f32(0.0))
    esi = np.where(valid, esi, f32(0.0))
    qvsw = np.zeros_like(p)
    qvsi = np.zeros_like(p)
    np.divide(ep_2 * esw, p - esw, out=qvsw, where=valid & ((p - esw) > f32(1.0)))
    np.divide(ep_2 * esi, p - esi, out=qvsi, where=valid & ((p - esi) > f32(1.0)))
    qcld = qi + qc + qs
    w = np.zeros_like(qcld)
    np.divide(qi + qs, qcld, out=w, where=qcld >= qcldmin)
    qvs = (f32(1.0) - w) * qvsw + w * qvsi
    rhum = np.zeros_like(qv)
    np.divide(qv, qvs, out=rhum, where=valid & (qvs > f32(0.0)))
    subsat = np.maximum(f32(1.0e-10), rhgrid * qvs - qv)
    arg = np.maximum(f32(-6.9), -alpha0 * qcld / subsat ** gamma)
    partial = (np.maximum(f32(1.0e-10), rhum) / rhgrid) ** pexp * (f32(1.0) - np.exp(arg).astype(np.float32))
    partial = np.where(partial < f32(0.01), f32(0.0), partial)
    out = np.where(valid & (qcld >= qcldmin), np.where(rhum >= rhgrid, f32(1.0), partial), f32(0.0))
    return np.ascontiguousarray(out.astype(np.float32))


def cal_cldfra1_parts(qv, qc, qi, qs, t, p) -> tuple[np.ndarray, np.ndarray]:
    """(rhum, partial before its 0.01 cut) of cal_cldfra1, for locating threshold cases."""
    qv, qc, qi, qs, t, p = (np.asarray(a, np.float32) for a in (qv, qc, qi, qs, t, p))
    with np.errstate(all="ignore"):
        ts = np.where((t > f32(100.0)) & (p > f32(100.0)), t, f32(273.15))
        tc = ts - f32(273.15)
        esw = f32(1000.0) * f32(0.61078) * np.exp(f32(17.2693882) * tc / (ts - f32(35.86)))
        esi = f32(1000.0) * f32(0.61078) * np.exp(f32(21.8745584) * tc / (ts - f32(7.66)))
        qvsw = np.where(p - esw > 1, f32(287.0 / 461.6) * esw / (p - esw), f32(0.0))
        qvsi = np.where(p - esi > 1, f32(287.0 / 461.6) * esi / (p - esi), f32(0.0))
        qcld = qi + qc + qs
        w = np.where(qcld >= f32(1e-12), (qi + qs) / qcld, f32(0.0))
        qvs = (f32(1.0) - w) * qvsw + w * qvsi
        rhum = np.where(qvs > 0, qv / qvs, f32(0.0))
        subsat = np.maximum(f32(1.0e-10), qvs - qv)
        arg = np.maximum(f32(-6.9), -f32(100.0) * qcld / subsat ** f32(0.49))
        partial = np.maximum(f32(1.0e-10), rhum) ** f32(0.25) * (f32(1.0) - np.exp(arg))
    return rhum.astype(np.float32), partial.astype(np.float32)


# ---------------------------------------------------------------------------
# cos zenith
# ---------------------------------------------------------------------------
def _xor_bits(v: np.ndarray, bits) -> np.ndarray:
    return np.bitwise_xor(np.asarray(v, np.float32).view(np.uint32), np.asarray(bits, np.uint32)).view(np.float32)


_INV_PI, _ROUND, _HALF_PI, _HALF = 0x3EA2F983, 0x4B400000, 0x3FC90FDB, 0x3F000000
_PI_PARTS = (0x40490000, 0x3A7DA000, 0x34222000, 0x2CB4611A)
_POLY = (0x362EDEF8, 0xB94FB7FF, 0x3C08876A, 0xBE2AAAA6)
_LIMIT = 0x461C4000


def _svml_core(src: np.ndarray, y: np.ndarray, octant: np.ndarray) -> np.ndarray:
    """Shared tail of the SVML kernels: 4-part pi reduction and the odd polynomial."""
    x = src - y * _bits32(_PI_PARTS[0])
    x = x - y * _bits32(_PI_PARTS[1])
    x = x - y * _bits32(_PI_PARTS[2])
    x = x - y * _bits32(_PI_PARTS[3])
    x2 = x * x
    sx = _xor_bits(x, octant)
    q = _bits32(_POLY[0]) * x2
    q = q + _bits32(_POLY[1])
    q = q * x2
    q = q + _bits32(_POLY[2])
    q = q * x2
    q = q + _bits32(_POLY[3])
    corr = x2 * q
    corr = sx * corr
    return sx + corr


def _octant(y: np.ndarray) -> np.ndarray:
    return np.left_shift(np.asarray(y, np.float32).view(np.uint32), np.uint32(31))


def svml_sinf(v: np.ndarray) -> np.ndarray:
    """Four-lane SVML sinf as runtime.py:6027-6060 restates it (binary32 steps)."""
    src = np.asarray(v, np.float32)
    bits = src.view(np.uint32)
    sign = np.bitwise_and(bits, np.uint32(0x80000000))
    a = np.bitwise_and(bits, np.uint32(0x7FFFFFFF)).view(np.float32)
    y = a * _bits32(_INV_PI)
    y = y + _bits32(_ROUND)
    octant = _octant(y)
    y = y - _bits32(_ROUND)
    r = _xor_bits(_svml_core(a, y, octant), sign)
    return np.where(np.abs(src) > _bits32(_LIMIT), np.sin(src), r).astype(np.float32)


def svml_cosf(v: np.ndarray) -> np.ndarray:
    """Four-lane SVML cosf as runtime.py:6063-6096 restates it (binary32 steps)."""
    src = np.asarray(v, np.float32)
    y = _bits32(_HALF_PI) + src
    y = y * _bits32(_INV_PI)
    y = y + _bits32(_ROUND)
    octant = _octant(y)
    y = y - _bits32(_ROUND)
    y = y - _bits32(_HALF)
    r = _svml_core(src, y, octant)
    return np.where(np.abs(src) > _bits32(_LIMIT), np.cos(src), r).astype(np.float32)


_libm = None


def _libm_trig(v: np.ndarray, cosine: bool) -> np.ndarray:
    """Scalar glibc sinf/cosf element by element (runtime.py:6099-6119)."""
    global _libm
    if _libm is None:
        lib = ctypes.CDLL(ctypes.util.find_library("m") or None)
        for name in ("sinf", "cosf"):
            fn = getattr(lib, name)
            fn.argtypes = (ctypes.c_float,)
            fn.restype = ctypes.c_float
        _libm = lib
    fn = _libm.cosf if cosine else _libm.sinf
    src = np.asarray(v, np.float32)
    return np.fromiter((fn(float(e)) for e in src.flat), np.float32, src.size).reshape(src.shape)


def coszen_scalars(julian: float, xtime: float, gmt: float, declin: float) -> tuple[float, float, float]:
    """Per-call scalars of calc_coszen: (gmt + local-time offset [h], sin declin, cos declin)."""
    da = f32(f32(f32(6.2831853071795862) * f32(f32(julian) - f32(1.0))) / f32(365.0))
    da2 = f32(f32(2.0) * da)
    eot = f32(0.000075)
    eot = f32(eot + f32(f32(0.001868) * f32(np.cos(da))))
    eot = f32(eot - f32(f32(0.032077) * f32(np.sin(da))))
    eot = f32(eot - f32(f32(0.014615) * f32(np.cos(da2))))
    eot = f32(eot - f32(f32(0.04089) * f32(np.sin(da2))))
    eot = f32(eot * f32(229.18))
    xt24 = f32(f32(np.fmod(f32(xtime), f32(1440.0))) + eot)
    t0 = f32(f32(gmt) + f32(xt24 / f32(60.0)))
    return float(t0), float(f32(np.sin(f32(declin)))), float(f32(np.cos(f32(declin))))


def calc_coszen(xlat, xlong, *, julian: float, xtime: float, gmt: float, declin: float) -> np.ndarray:
    """cos(solar zenith) on (nx, ny) float32 grids (runtime.py:6207-6243)."""
    degrad = f32(np.pi / 180.0)
    lat = np.asarray(xlat, np.float32)
    lon = np.asarray(xlong, np.float32)
    t0, sd, cd = (f32(v) for v in coszen_scalars(julian, xtime, gmt, declin))
    tloc = t0 + lon / f32(15.0)
    hrang = (f32(15.0) * (tloc - f32(12.0))) * degrad
    xxlat = lat * degrad
    stop = (xxlat.shape[0] // 4) * 4
    s_lat, c_lat, c_hr = svml_sinf(xxlat), svml_cosf(xxlat), svml_cosf(hrang)
    if stop < xxlat.shape[0]:
        s_lat[stop:] = _libm_trig(xxlat[stop:], cosine=False)
        c_lat[stop:] = _libm_trig(xxlat[stop:], cosine=True)
        c_hr[stop:] = _libm_trig(hrang[stop:], cosine=True)
    cz = s_lat * sd + (c_lat * cd) * c_hr
    return np.ascontiguousarray(np.minimum(np.maximum(cz, f32(-1.0)), f32(1.0)).astype(np.float32))


# ---------------------------------------------------------------------------
# CAM ozone
# ---------------------------------------------------------------------------
def cam_o3rad(xlat, p3d, *, julian: float, plev, lat_oz, ozone) -> np.ndarray:
    """Ozone volume mixing ratio on (nx, nk, ny) from a CAM climatology (runtime.py:5753-5801).

    ``plev`` (levsiz,) Pa ascending, ``lat_oz`` (latsiz,) degrees ascending,
    ``ozone`` (12, latsiz, levsiz)."""
    plev = np.asarray(plev, np.float32)
    lat_oz = np.asarray(lat_oz, np.float32)
    ozone = np.asarray(ozone, np.float32)
    m0, m1, w1, w2 = ozone_month_weights(julian)
    p = np.asarray(p3d, np.float32)
    nx, nk, ny = p.shape
    nlev = plev.shape[0]
    lat = np.asarray(xlat, np.float32).reshape(-1)
    li = np.clip(np.searchsorted(lat_oz, lat, side="left") - 1, 0, lat_oz.size - 2)
    dlat = (lat - lat_oz[li]).astype(np.float32)
    span = (lat_oz[li + 1] - lat_oz[li]).astype(np.float32)
    per_month = []
    for m in (m0, m1):
        lo, hi = ozone[m, li, :], ozone[m, li + 1, :]
        slope = ((hi - lo).astype(np.float32) / span[:, None]).astype(np.float32)
        per_month.append((lo + (slope * dlat[:, None]).astype(np.float32)).astype(np.float32))
    prof = ((per_month[0] * f32(w1)).astype(np.float32)
            + (per_month[1] * f32(w2)).astype(np.float32)).astype(np.float32).reshape(nx, ny, nlev)
    pk = np.transpose(p, (0, 2, 1))
    k = np.clip(np.searchsorted(plev, p, side="left") - 1, 0, nlev - 2).transpose(0, 2, 1)
    o_lo = np.take_along_axis(prof, k, axis=2)
    o_hi = np.take_along_axis(prof, k + 1, axis=2)
    dpu = (pk - plev[k]).astype(np.float32)
    dpl = (plev[k + 1] - pk).astype(np.float32)
    out = (((o_lo * dpl).astype(np.float32) + (o_hi * dpu).astype(np.float32)).astype(np.float32)
           / (dpl + dpu).astype(np.float32)).astype(np.float32)
    top = (((prof[:, :, :1] * pk).astype(np.float32)) / plev[0]).astype(np.float32)
    out = np.where(pk < plev[0], top, out)
    out = np.where(pk > plev[-1], prof[:, :, -1:], out)
    return np.ascontiguousarray(np.transpose(out, (0, 2, 1)).astype(np.float32))
