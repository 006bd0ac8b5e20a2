"""Seeded synthetic WRF column states for the RRTMG radiation calls.

No public dataset is involved: the reference validates only against WRF
``wrfout`` files of a case directory that is not shipped.  These generators
produce model-domain inputs in the reference's runtime layout, 3-D fields as
``(west_east, bottom_top, south_north)`` float32 and 2-D fields as
``(west_east, south_north)`` (the layout documented at
``src/wrf_jax/physics/module_ra_rrtmg_sw.py:2435-2438``).

Profile recipe (identical for every workload, only the spreads change):

* surface pressure U(950, 1030) hPa, model top ``p_top`` = 50 hPa, interfaces
  from a stretched hybrid-eta curve (denser near the ground);
* temperature 288 K lapsing at 6.5 K/km (standard-atmosphere pressure form)
  to the 200 hPa tropopause, isothermal above, plus N(0, ``t_noise``) per level;
* water vapour = RH x saturation (Tetens), RH ~ U(``rh_lo``, 1), decaying with
  height through the saturation curve;
* ozone as a volume mixing ratio, a log-pressure Gaussian peaking at 8 ppmv
  near 10 hPa over a 30 ppbv floor;
* cloud fraction Bernoulli(``cloud_p``) per level below 300 hPa, with
  qc ~ U(0, 5e-4), qi ~ U(0, 2e-4) kg/kg where cloudy (qs = 0);
* surface albedo U(0.05, 0.4), emissivity U(0.9, 1.0), skin temperature =
  lowest-level T + U(-3, 3) K, all land (xland = 1), no ice or snow;
* cosine of the solar zenith U(0, 1) with ``night_fraction`` of columns at 0.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

R_DRY = 287.0
CP_DRY = 1004.5
P_TOP_PA = 5000.0

# Greenhouse-gas volume mixing ratios (WRF RRTMG defaults, runtime.py:5658-5664)
GASES = dict(co2vmr=410.0e-6, n2ovmr=319.0e-9, ch4vmr=1774.0e-9,
             cfc11vmr=0.251e-9, cfc12vmr=0.538e-9)


@dataclass
class ColumnState:
    """One synthetic model domain: arrays keyed by the reference keyword names."""

    fields: dict
    scalars: dict
    nx: int
    ny: int
    nk: int

    def lw_kwargs(self) -> dict:
        f = self.fields
        keys = ("p3d", "p8w", "pi3d", "t3d", "t8w", "tsk", "dz8w", "qv3d", "qc3d",
                "qi3d", "qs3d", "cldfra3d", "o33d", "emiss", "xland", "xice", "snow",
                "re_cloud", "re_ice", "re_snow")
        kw = {k: f[k] for k in keys}
        kw.update(p_top=self.scalars["p_top"], yr=self.scalars["yr"],
                  julian=self.scalars["julian"], **{k: self.scalars[k] for k in GASES})
        kw.update(has_reqc=self.scalars["has_reqc"], has_reqi=self.scalars["has_reqi"],
                  has_reqs=self.scalars["has_reqs"], icloud=1, cldovrlp=2)
        return kw

    def sw_kwargs(self) -> dict:
        f = self.fields
        keys = ("p3d", "p8w", "pi3d", "t3d", "t8w", "tsk", "dz8w", "qv3d", "qc3d",
                "qi3d", "qs3d", "cldfra3d", "o33d", "albedo", "coszr", "xland", "xice",
                "snow", "re_cloud", "re_ice", "re_snow")
        kw = {k: f[k] for k in keys}
        kw.update(solcon=self.scalars["solcon"], yr=self.scalars["yr"],
                  julian=self.scalars["julian"],
                  co2vmr=self.scalars["co2vmr"], n2ovmr=self.scalars["n2ovmr"],
                  ch4vmr=self.scalars["ch4vmr"])
        kw.update(has_reqc=self.scalars["has_reqc"], has_reqi=self.scalars["has_reqi"],
                  has_reqs=self.scalars["has_reqs"], icloud=1, cldovrlp=2)
        return kw


def eccentricity_factor(julian: float) -> float:
    """Earth-Sun distance factor (Spencer 1971 Fourier series) in float32."""
    f = np.float32
    rjul = f(f(f(julian) * f(360.0)) / f(365.0)) * f(np.pi / 180.0)
    ecc = f(1.000110) + f(0.034221) * f(np.cos(rjul)) + f(0.001280) * f(np.sin(rjul))
    ecc = ecc + f(0.000719) * f(np.cos(2 * rjul)) + f(0.000077) * f(np.sin(2 * rjul))
    return float(f(ecc))


def _eta_interfaces(nk: int) -> np.ndarray:
    s = np.linspace(0.0, 1.0, nk + 1)
    a = 3.0
    return (np.exp(-a * s) - np.exp(-a)) / (1.0 - np.exp(-a))  # 1 at the surface, 0 at the top


def _qsat(t: np.ndarray, p_pa: np.ndarray) -> np.ndarray:
    es = 610.78 * np.exp(17.27 * (t - 273.16) / (t - 35.86))
    es = np.minimum(es, 0.5 * p_pa)
    return 0.622 * es / (p_pa - 0.378 * es)


def make_columns(nx: int, ny: int, nk: int, *, seed: int = 0, t_noise: float = 2.0,
                 rh_lo: float = 0.2, cloud_p: float | tuple = 0.3,
                 night_fraction: float = 0.3, has_req: bool = False,
                 fractional_clouds: bool = False, p_top: float = P_TOP_PA,
                 julian: float = 172.5, yr: int = 2024) -> ColumnState:
    """Generate one domain of nx x ny columns with nk mass levels."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ncol = nx * ny
    psfc = rng.uniform(950.0e2, 1030.0e2, size=ncol)
    eta = _eta_interfaces(nk)
    p8w = p_top + eta[None, :] * (psfc[:, None] - p_top)              # (ncol, nk+1) Pa
    p8w[:, nk] = p_top
    p3d = 0.5 * (p8w[:, :-1] + p8w[:, 1:])                              # (ncol, nk)

    def t_profile(p_pa):
        t = 288.0 * (np.maximum(p_pa, 200.0e2) / 101325.0) ** (R_DRY * 0.0065 / 9.80665)
        return t

    t3d = t_profile(p3d) + rng.normal(0.0, t_noise, size=(ncol, nk))
    t8w = np.empty((ncol, nk + 1))
    t8w[:, 1:nk] = 0.5 * (t3d[:, :-1] + t3d[:, 1:])
    t8w[:, 0] = t3d[:, 0] + (t3d[:, 0] - t8w[:, 1])
    t8w[:, nk] = t3d[:, nk - 1]
    tsk = t3d[:, 0] + rng.uniform(-3.0, 3.0, size=ncol)

    rh = rng.uniform(rh_lo, 1.0, size=(ncol, nk))
    qv = rh * _qsat(t3d, p3d)

    p_hpa = p3d / 100.0
    o3 = 8.0e-6 * np.exp(-0.5 * (np.log(p_hpa / 10.0) / 1.1) ** 2) + 3.0e-8

    if isinstance(cloud_p, tuple):
        col_p = rng.uniform(cloud_p[0], cloud_p[1], size=(ncol, 1))
    else:
        col_p = np.full((ncol, 1), float(cloud_p))
    cloudy = (rng.uniform(size=(ncol, nk)) < col_p) & (p3d > 300.0e2)
    cldfra = cloudy.astype(np.float64)
    if fractional_clouds:
        cldfra = np.where(cloudy, rng.uniform(0.05, 1.0, size=(ncol, nk)), 0.0)
    qc = np.where(cloudy, rng.uniform(0.0, 5.0e-4, size=(ncol, nk)), 0.0)
    qi = np.where(cloudy, rng.uniform(0.0, 2.0e-4, size=(ncol, nk)), 0.0)
    qs = np.zeros((ncol, nk))

    albedo = rng.uniform(0.05, 0.4, size=ncol)
    emiss = rng.uniform(0.9, 1.0, size=ncol)
    coszr = rng.uniform(0.0, 1.0, size=ncol)
    coszr[rng.uniform(size=ncol) < night_fraction] = 0.0

    if has_req:
        re_cloud = rng.uniform(2.5e-6, 20.0e-6, size=(ncol, nk))
        re_ice = rng.uniform(5.0e-6, 100.0e-6, size=(ncol, nk))
        re_snow = rng.uniform(10.0e-6, 200.0e-6, size=(ncol, nk))
    else:
        re_cloud = np.zeros((ncol, nk))
        re_ice = np.zeros((ncol, nk))
        re_snow = np.zeros((ncol, nk))

    pi3d = (p3d / 1.0e5) ** (R_DRY / CP_DRY)
    dz8w = np.full((ncol, nk), 250.0)

    def to3d(a):  # (ncol, nz) -> (nx, nz, ny)
        nz = a.shape[1]
        return np.ascontiguousarray(np.asarray(a, np.float32).reshape(nx, ny, nz).transpose(0, 2, 1))

    def to2d(a):
        return np.ascontiguousarray(np.asarray(a, np.float32).reshape(nx, ny))

    fields = dict(
        p3d=to3d(p3d), p8w=to3d(p8w), pi3d=to3d(pi3d), t3d=to3d(t3d), t8w=to3d(t8w),
        tsk=to2d(tsk), dz8w=to3d(dz8w), qv3d=to3d(qv), qc3d=to3d(qc), qi3d=to3d(qi),
        qs3d=to3d(qs), cldfra3d=to3d(cldfra), o33d=to3d(o3), emiss=to2d(emiss),
        albedo=to2d(albedo), coszr=to2d(coszr), xland=to2d(np.ones(ncol)),
        xice=to2d(np.zeros(ncol)), snow=to2d(np.zeros(ncol)), re_cloud=to3d(re_cloud),
        re_ice=to3d(re_ice), re_snow=to3d(re_snow),
    )
    h = 1 if has_req else 0
    scalars = dict(p_top=float(p_top), yr=yr, julian=julian,
                   solcon=float(np.float32(1370.0) * np.float32(eccentricity_factor(julian))),
                   has_reqc=h, has_reqi=h, has_reqs=h, **GASES)
    return ColumnState(fields=fields, scalars=scalars, nx=nx, ny=ny, nk=nk)



def lat_lon(nx: int, ny: int, *, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """(xlat, xlong) in degrees on an (nx, ny) grid: latitudes U(-90, 90) and
    longitudes U(-180, 180), float32."""
    rng = np.random.default_rng(seed + 1000)
    lat = rng.uniform(-90.0, 90.0, (nx, ny)).astype(np.float32)
    lon = rng.uniform(-180.0, 180.0, (nx, ny)).astype(np.float32)
    return lat, lon


def cam_ozone_climatology(*, seed: int = 0, levsiz: int = 59, latsiz: int = 64):
    """Seeded stand-in for a case's CAM ozone files (ozone_plev.formatted,
    ozone_lat.formatted, ozone.formatted): ``levsiz`` pressure levels in hPa,
    geometric from 0.35 to 1000 hPa; ``latsiz`` latitudes evenly spaced
    within +-87.9 degrees; (12, latsiz, levsiz) volume mixing ratios, a
    log-pressure Gaussian of 2-10 ppmv near 10 hPa varying with latitude and
    month over a 20 ppbv floor, with 5 % multiplicative noise."""
    rng = np.random.default_rng(seed + 2000)
    plev = np.geomspace(0.35, 1000.0, levsiz).astype(np.float32)
    lat = np.linspace(-87.9, 87.9, latsiz).astype(np.float32)
    month = np.arange(12)[:, None, None]
    phi = np.deg2rad(lat)[None, :, None]
    lp = np.log(plev.astype(np.float64))[None, None, :]
    peak = 6.0e-6 + 3.0e-6 * np.cos(phi) ** 2 + 1.0e-6 * np.sin(phi) * np.cos(2 * np.pi * month / 12)
    oz = 2.0e-8 + peak * np.exp(-0.5 * ((lp - np.log(10.0)) / 1.1) ** 2)
    oz *= rng.uniform(0.95, 1.05, oz.shape)
    return plev, lat, oz.astype(np.float32)


def write_cam_ozone_files(directory, plev_hpa, lat, ozone) -> None:
    """Write a climatology in the three text files of a WRF case directory
    (values exact in binary32: nine significant digits; one row per month and
    latitude)."""
    from pathlib import Path
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    np.savetxt(d / "ozone_plev.formatted", np.asarray(plev_hpa, np.float32), fmt="%.9e")
    np.savetxt(d / "ozone_lat.formatted", np.asarray(lat, np.float32), fmt="%.9e")
    np.savetxt(d / "ozone.formatted", np.asarray(ozone, np.float32).reshape(-1, np.shape(ozone)[-1]), fmt="%.9e")

# Named workloads (grid sizes and spreads).
WORKLOADS = {
    "cpu_64x64x44": dict(nx=64, ny=64, nk=44, seed=0),
    "plain_425x425x50": dict(nx=425, ny=425, nk=50, seed=0),
    "training_2m_x50": dict(nx=2000, ny=1000, nk=50, seed=1, t_noise=4.0, rh_lo=0.05,
                            cloud_p=(0.0, 0.6)),
    "inference_1000x1000x50": dict(nx=1000, ny=1000, nk=50, seed=2),
}
