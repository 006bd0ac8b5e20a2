"""FP64 mode on the GPU (rrtmg_config.fp64_steps = 1) against the oracle's
FP64 mode: bit for bit.  The two binary64 steps (SW reftra of layers whose
delta-scaled single-scattering albedo is >= 0.999 or whose optical depth is
below 0.1, and the heating rates of the five highest model layers) are IEEE
binary64 operations in the same order on both sides, rounded once to
binary32."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import case_kwargs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rrtmg(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import rrtmg as mod
    return mod


def _assert_fields(got, ref: dict, tag: str) -> None:
    for name, value in ref.items():
        np.testing.assert_array_equal(np.asarray(getattr(got, name)), value, err_msg=f"{tag} {name}")


@pytest.mark.parametrize("case", ("c0_4x4x44", "req_3x3x44", "fraccloud_ptop10_3x3x30", "overcast_2x2x40",
                                  "odd_1x3x17"))
def test_fp64_mode_golden_inputs(rrtmg, oracle, golden, case):
    for side in ("lw", "sw"):
        kw = case_kwargs(golden[case], side)
        fn = rrtmg.rrtmg_lwrad_wrf_columns if side == "lw" else rrtmg.rrtmg_swrad_wrf_columns
        want = (oracle.lwrad if side == "lw" else oracle.swrad)(fp64_steps=1, **kw)
        _assert_fields(fn(fp64_steps=True, **kw), want, f"{case} {side}")


@pytest.mark.parametrize("nx,ny,nk,seed,extra", [
    (64, 64, 44, 0, {}),
    (17, 23, 50, 1, dict(fractional_clouds=True)),
    (9, 40, 60, 2, dict(has_req=True, cloud_p=0.6)),
    (200, 200, 50, 3, dict(fractional_clouds=True)),
])
def test_fp64_mode_random_domains(rrtmg, oracle, pkg, nx, ny, nk, seed, extra):
    from wrf_jax_b200 import synthetic
    st = synthetic.make_columns(nx, ny, nk, seed=seed, **extra)
    _assert_fields(rrtmg.rrtmg_lwrad_wrf_columns(fp64_steps=True, **st.lw_kwargs()),
                   oracle.lwrad(fp64_steps=1, **st.lw_kwargs()), "lw")
    _assert_fields(rrtmg.rrtmg_swrad_wrf_columns(fp64_steps=True, **st.sw_kwargs()),
                   oracle.swrad(fp64_steps=1, **st.sw_kwargs()), "sw")
