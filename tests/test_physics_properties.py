"""Physical properties of the radiation path, checked on the CPU oracle (which
the CUDA path reproduces bit for bit; the GPU leg of each test runs the same
inputs through the C-ABI and requires the oracle's bits):

* energy identity: the column-integrated heating equals the net flux
  convergence, sum_l hr_l dp_l / heatfac = F_net(bottom) - F_net(top), since
  hr_l = heatfac (F_net(l) - F_net(l+1)) / dp_l (lw:5706-5709, sw:2285-2300);
* an isothermal atmosphere over a black surface at the same temperature
  radiates nearly the same upward flux at every level: each band's Planck
  radiance is the same everywhere, and only its split among the band's
  g-points (the Planck fractions, which follow each layer's gas ratios)
  varies from layer to layer;
* without cloud every all-sky result equals its clear-sky counterpart bit for
  bit, and the SW model-top downward flux is the incoming beam solcon *
  coszen, of which the column absorbs a positive share.
"""

from __future__ import annotations

import numpy as np
import pytest

HEATFAC = (9.8066 * 8.64e4) / (1004.5 * 1.0e2)


@pytest.fixture(scope="module")
def domain(pkg):
    from wrf_jax_b200 import synthetic
    return synthetic.make_columns(8, 6, 50, seed=12, fractional_clouds=True, night_fraction=0.25)


def _columns(a):  # (nx, nz, ny) -> (ncol, nz)
    a = np.asarray(a, np.float64)
    return np.swapaxes(a, 1, 2).reshape(-1, a.shape[1])


def test_energy_identity_lw(oracle, domain):
    kw = domain.lw_kwargs()
    d = oracle.lwrad(diagnostics=True, **kw)["diag"]
    nk = kw["t3d"].shape[1]
    plev = _columns(kw["p8w"]) / 100.0                       # model interfaces, hPa
    hr = np.asarray(d["hr"], np.float64)[:, :nk]             # K/day
    fnet = np.asarray(d["uflx"], np.float64) - np.asarray(d["dflx"], np.float64)
    lhs = (hr * (plev[:, :-1] - plev[:, 1:])).sum(axis=1) / HEATFAC
    rhs = fnet[:, 0] - fnet[:, nk]
    np.testing.assert_allclose(lhs, rhs, rtol=2e-4, atol=2e-3)


def test_energy_identity_sw(oracle, domain):
    kw = domain.sw_kwargs()
    d = oracle.swrad(diagnostics=True, **kw)["diag"]
    nk = kw["t3d"].shape[1]
    day = (np.asarray(kw["coszr"]) > 0).reshape(-1)
    plev = _columns(kw["p8w"]) / 100.0
    hr = np.asarray(d["hr"], np.float64)[:, :nk]
    # SW net flux is down minus up; the levels run bottom-up
    fnet = np.asarray(d["dflx"], np.float64) - np.asarray(d["uflx"], np.float64)
    lhs = (hr * (plev[:, :-1] - plev[:, 1:])).sum(axis=1) / HEATFAC
    rhs = fnet[:, nk] - fnet[:, 0]
    assert day.sum() >= 20
    np.testing.assert_allclose(lhs[day], rhs[day], rtol=2e-4, atol=2e-3)


def _isothermal(domain, t0=260.0):
    st = domain
    f = {k: v.copy() for k, v in st.fields.items()}
    for k in ("t3d", "t8w"):
        f[k][...] = t0
    f["tsk"][...] = t0
    f["emiss"][...] = 1.0
    for k in ("qc3d", "qi3d", "qs3d", "cldfra3d"):
        f[k][...] = 0.0
    kw = st.lw_kwargs()
    kw.update({k: f[k] for k in kw if k in f})
    return kw


def test_isothermal_black_column_has_constant_upward_flux(oracle, domain):
    kw = _isothermal(domain)
    d = oracle.lwrad(diagnostics=True, **kw)["diag"]
    nk = kw["t3d"].shape[1]
    up = np.asarray(d["uflx"], np.float64)[:, : nk + 1]      # surface to the model top
    np.testing.assert_allclose(up, up[:, :1] * np.ones_like(up), rtol=5e-3)
    # and it is the band-integrated Planck flux: close to sigma T^4 (the bands
    # cover 10-3250 cm-1, nearly the whole spectrum at 260 K)
    sigma_t4 = 5.670374e-8 * 260.0 ** 4
    assert np.all(np.abs(up[:, 0] / sigma_t4 - 1.0) < 0.01)


def _clear(domain):
    st = domain
    f = {k: v.copy() for k, v in st.fields.items()}
    for k in ("qc3d", "qi3d", "qs3d", "cldfra3d"):
        f[k][...] = 0.0
    return f


def test_cloudless_columns_equal_their_clear_sky_results(oracle, domain):
    """Without condensate and cloud fraction every all-sky result equals its
    clear-sky counterpart bit for bit (the McICA columns are all clear)."""
    f = _clear(domain)
    kw = domain.lw_kwargs()
    kw.update({k: f[k] for k in kw if k in f})
    r = oracle.lwrad(**kw)
    for a, b in (("rthratenlw", "rthratenlwc"), ("lwupt", "lwuptc"), ("lwupb", "lwupbc"), ("lwdnb", "lwdnbc")):
        np.testing.assert_array_equal(r[a], r[b], err_msg=a)
    kw = domain.sw_kwargs()
    kw.update({k: f[k] for k in kw if k in f})
    r = oracle.swrad(**kw)
    for a, b in (("rthratensw", "rthratenswc"), ("swupt", "swuptc"), ("swupb", "swupbc"), ("swdnb", "swdnbc"),
                 ("swddir", "swddirc")):
        np.testing.assert_array_equal(r[a], r[b], err_msg=a)
    assert np.all(r["swcf"] == 0)


def test_incoming_solar_flux_and_column_energy_balance(oracle, domain):
    """The model-top downward flux is the incoming beam, solcon * coszen (the
    reference spectrum's bands sum to the solar constant it is scaled by);
    the column absorbs a positive share of it below that."""
    kw = domain.sw_kwargs()
    r = oracle.swrad(**kw)
    mu = np.asarray(kw["coszr"], np.float64)
    day = mu > 0
    top = np.asarray(r["swdnt"], np.float64)
    np.testing.assert_allclose(top[day], kw["solcon"] * mu[day], rtol=2e-3)
    absorbed = (top - np.asarray(r["swupt"], np.float64)) - (np.asarray(r["swdnb"], np.float64) -
                                                              np.asarray(r["swupb"], np.float64))
    assert np.all(absorbed[day] > 0) and np.all(absorbed[day] < 0.5 * top[day])
    for name in ("swdnt", "swupt", "swdnb", "swupb", "gsw", "swddir"):
        assert np.all(np.asarray(r[name])[~day] == 0), name


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["isothermal", "cloudless"])
def test_gpu_matches_oracle_on_limit_inputs(oracle, domain, case):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import rrtmg
    if case == "isothermal":
        kw = _isothermal(domain)
        got, want = rrtmg.rrtmg_lwrad_wrf_columns(**kw), oracle.lwrad(**kw)
    else:
        f = _clear(domain)
        kw = domain.sw_kwargs()
        kw.update({k: f[k] for k in kw if k in f})
        got, want = rrtmg.rrtmg_swrad_wrf_columns(**kw), oracle.swrad(**kw)
    for name, value in want.items():
        np.testing.assert_array_equal(np.asarray(getattr(got, name)), value, err_msg=f"{case} {name}")
