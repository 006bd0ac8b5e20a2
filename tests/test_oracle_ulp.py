"""How much a last-place libm difference moves the LW outputs.

The reference computes two LW results with XLA's binary32 libm instead of the
glibc algorithms it emulates elsewhere: the cloud absorptance
``1 - exp(-odcld)`` (module_ra_rrtmg_lw.py:5564) and the minor-gas scaling
power (module_ra_rrtmg_lw.py:134-144).  The oracle and the kernels use glibc
``expf``/``powf`` there, and XLA's results may differ from glibc's by one ulp.
This test moves each result by +-1 ulp in the oracle (a test knob,
``ora_set_libm_perturbation``) and bounds the change of every LW output:

* fluxes (the 2-D outputs): at most 1e-4 W/m2, ten times inside the
  1e-3 W/m2 parity tolerance;
* heating (rthratenlw/c converted to K/day): at most 2e-4 K/day.  One ulp of
  a 300-400 W/m2 flux is 3.05e-5 W/m2, and the heating of a layer is
  (g * 86400 / (cp * 100)) * dF / dp = 8.435 * dF / dp(hPa), so in the
  thinnest model layers near a 50 hPa top (a few hPa) a one-ulp change of
  both bounding fluxes is already about 1e-4 K/day: a 1e-4
  K/day heating tolerance is at the binary32 resolution of the fluxes there.

The measured maxima are printed (pytest -s).
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

FLUX_2D = ("lwupt", "lwuptc", "lwdnt", "lwdntc", "lwupb", "lwupbc", "lwdnb", "lwdnbc", "glw", "olr", "lwcf")
FLUX_BOUND = 1.0e-4   # W/m2
HEAT_BOUND = 2.0e-4   # K/day


@pytest.fixture(scope="module")
def knob(oracle):
    fn = oracle.lib.ora_set_libm_perturbation
    fn.argtypes = [ctypes.c_int, ctypes.c_int]
    fn.restype = None
    yield fn
    fn(0, 0)


@pytest.mark.parametrize("extra", [{}, dict(fractional_clouds=True), dict(has_req=True, cloud_p=0.6)],
                         ids=["binary-clouds", "fractional-clouds", "effective-radii"])
def test_one_ulp_libm_difference_bound(pkg, oracle, knob, extra):
    from wrf_jax_b200 import synthetic
    st = synthetic.make_columns(40, 40, 50, seed=5, **extra)
    kw = st.lw_kwargs()
    pi3d = np.asarray(kw["pi3d"], np.float64)
    base = oracle.lwrad(**kw)
    worst = {}
    for exp_ulps, pow_ulps in ((1, 0), (-1, 0), (0, 1), (0, -1)):
        knob(exp_ulps, pow_ulps)
        try:
            r = oracle.lwrad(**kw)
        finally:
            knob(0, 0)
        dheat = max(float(np.abs((r[k].astype(np.float64) - base[k]) * 86400.0 * pi3d).max())
                    for k in ("rthratenlw", "rthratenlwc"))
        dflux = max(float(np.abs(r[k].astype(np.float64) - base[k]).max()) for k in FLUX_2D)
        worst[(exp_ulps, pow_ulps)] = (dheat, dflux)
        assert dflux <= FLUX_BOUND, (exp_ulps, pow_ulps, dflux)
        assert dheat <= HEAT_BOUND, (exp_ulps, pow_ulps, dheat)
    # the perturbation must actually reach the outputs (the knob is live)
    assert max(v[0] for v in worst.values()) > 0.0
    print("\n+-1 ulp (exp, pow) -> max |d heating| K/day, max |d flux| W/m2:",
          {k: ("%.3g" % a, "%.3g" % b) for k, (a, b) in worst.items()})
