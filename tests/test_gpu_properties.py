"""Size-independent properties of the plain kernels on the full 425 x 425 x 50
domain (180,625 columns), where the CPU oracle would take minutes:

* the domain split into south-north halves (the multi-GPU partition) gives
  the whole-domain result bit for bit, LW and SW;
* night columns (cos zenith 0) have exactly zero shortwave outputs;
* shortwave outputs are homogeneous of degree one in the solar constant: the
  incident flux is scon / 1368.22 * sfluxzen * mu0 and every later step
  scales or sums it, so doubling scon doubles every output to within 1e-6 of
  the column's flux scale (most values exactly; the direct-beam sums differ
  in the last place for a few percent of the columns, and the diffuse flux,
  a difference of two fluxes, carries that absolute difference).
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def full(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import rrtmg, synthetic
    st = synthetic.make_columns(425, 425, 50, seed=0)
    return rrtmg, st


def test_row_halves_equal_the_whole_domain(full):
    from wrf_jax_b200 import sharding
    rrtmg, st = full
    for side, call, kw in (("lw", rrtmg.rrtmg_lwrad_wrf_columns, st.lw_kwargs()),
                           ("sw", rrtmg.rrtmg_swrad_wrf_columns, st.sw_kwargs())):
        whole = call(**kw)._asdict()
        halves = []
        for j0, j1 in sharding.batch_partitions(425, 1, 2):
            halves.append(call(**{k: sharding.slice_rows(v, 425, 425, j0, j1) for k, v in kw.items()})._asdict())
        for name, value in whole.items():
            joined = np.concatenate([h[name] for h in halves], axis=-1)
            np.testing.assert_array_equal(joined, value, err_msg=f"{side} {name}")


def test_night_columns_have_zero_shortwave(full):
    rrtmg, st = full
    kw = st.sw_kwargs()
    night = kw["coszr"] <= 0
    assert 0.2 < night.mean() < 0.4
    out = rrtmg.rrtmg_swrad_wrf_columns(**kw)._asdict()
    for name, value in out.items():
        if name == "coszr":
            continue
        v = np.transpose(value, (0, 2, 1))[night] if value.ndim == 3 else value[night]
        assert not np.any(v), name


def test_shortwave_is_linear_in_the_solar_constant(full):
    rrtmg, st = full
    kw = st.sw_kwargs()
    one = rrtmg.rrtmg_swrad_wrf_columns(**kw)._asdict()
    kw2 = dict(kw, solcon=2.0 * kw["solcon"])
    two = rrtmg.rrtmg_swrad_wrf_columns(**kw2)._asdict()
    for name, v1 in one.items():
        if name == "coszr":
            np.testing.assert_array_equal(two[name], v1)
            continue
        want = 2.0 * v1.astype(np.float64)
        err = np.abs(two[name].astype(np.float64) - want)
        # the column's scale: its largest value over levels (heating) or the
        # surface downward flux (2-D fluxes)
        scale = (np.max(np.abs(want), axis=1, keepdims=True) if want.ndim == 3
                 else np.maximum(np.abs(want), 2.0 * np.abs(one["swdnb"].astype(np.float64))))
        assert np.all(err <= 1e-6 * scale + 1e-30), name
