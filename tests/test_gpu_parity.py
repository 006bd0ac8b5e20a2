"""CUDA path (through the C-ABI) against the reference's golden fixtures and the
CPU oracle.  The bar is bit-exact binary32 equality: the kernels follow the
reference's operation order with per-operation rounding and glibc-identical
logf/expf, so any difference is a defect."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import case_kwargs

pytestmark = pytest.mark.gpu

CASES = ("c0_4x4x44", "c1_3x5x50", "req_3x3x44", "fraccloud_ptop10_3x3x30", "allnight_2x3x44",
         "clearsky_allday_3x2x44", "overcast_2x2x40", "icloud0_2x2x44", "odd_1x3x17", "sf8_3x4x44")


@pytest.fixture(scope="module")
def rrtmg(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import rrtmg as mod
    return mod


def _assert_fields(got, ref: dict, tag: str) -> None:
    for name, value in ref.items():
        g = np.asarray(getattr(got, name) if not isinstance(got, dict) else got[name])
        np.testing.assert_array_equal(g, value, err_msg=f"{tag} {name}")


@pytest.mark.parametrize("case", CASES)
def test_lw_matches_reference_golden(rrtmg, golden, case):
    got = rrtmg.rrtmg_lwrad_wrf_columns(**case_kwargs(golden[case], "lw"))
    _assert_fields(got, golden[case]["lw"], f"{case} lw")


@pytest.mark.parametrize("case", CASES)
def test_sw_matches_reference_golden(rrtmg, golden, case):
    got = rrtmg.rrtmg_swrad_wrf_columns(**case_kwargs(golden[case], "sw"))
    _assert_fields(got, golden[case]["sw"], f"{case} sw")


@pytest.mark.parametrize("nx,ny,nk,seed,extra", [
    (64, 64, 44, 0, {}),
    (17, 23, 50, 1, dict(fractional_clouds=True)),
    (9, 40, 60, 2, dict(has_req=True, cloud_p=0.6)),
    (33, 7, 24, 3, dict(p_top=2000.0, night_fraction=0.0)),
    # more than 4,096 columns: the one-thread-per-column SW schedule (smaller
    # domains above run the band-split schedule)
    (96, 64, 44, 4, dict(fractional_clouds=True)),
])
def test_random_domains_match_oracle(rrtmg, oracle, pkg, nx, ny, nk, seed, extra):
    from wrf_jax_b200 import synthetic
    st = synthetic.make_columns(nx, ny, nk, seed=seed, **extra)
    lw = rrtmg.rrtmg_lwrad_wrf_columns(**st.lw_kwargs())
    sw = rrtmg.rrtmg_swrad_wrf_columns(**st.sw_kwargs())
    _assert_fields(lw, oracle.lwrad(**st.lw_kwargs()), "lw")
    _assert_fields(sw, oracle.swrad(**st.sw_kwargs()), "sw")


def test_device_tensors_in_place(rrtmg, pkg):
    """torch CUDA tensors in, torch CUDA tensors out, equal to the host path."""
    import torch
    from wrf_jax_b200 import synthetic
    st = synthetic.make_columns(8, 8, 44, seed=5)
    host = rrtmg.rrtmg_lwrad_wrf_columns(**st.lw_kwargs())
    kw = {k: (torch.from_numpy(v).cuda() if isinstance(v, np.ndarray) else v) for k, v in st.lw_kwargs().items()}
    dev = rrtmg.rrtmg_lwrad_wrf_columns(**kw)
    for name in host._fields:
        t = getattr(dev, name)
        assert t.is_cuda
        np.testing.assert_array_equal(t.cpu().numpy(), getattr(host, name))


def test_unsupported_option_raises(rrtmg, pkg):
    from wrf_jax_b200 import synthetic
    st = synthetic.make_columns(2, 2, 10, seed=0)
    kw = st.lw_kwargs()
    kw["rounding_token"] = 1
    with pytest.raises(NotImplementedError):
        rrtmg.rrtmg_lwrad_wrf_columns(**kw)


def test_zero_rounding_token_is_a_plain_store(rrtmg, pkg):
    """The runtime always passes its uint32 token (0 in production)."""
    from wrf_jax_b200 import synthetic
    st = synthetic.make_columns(5, 4, 30, seed=9)
    plain_lw = rrtmg.rrtmg_lwrad_wrf_columns(**st.lw_kwargs())
    plain_sw = rrtmg.rrtmg_swrad_wrf_columns(**st.sw_kwargs())
    tok_lw = rrtmg.rrtmg_lwrad_wrf_columns(**st.lw_kwargs(), rounding_token=np.uint32(0))
    tok_sw = rrtmg.rrtmg_swrad_wrf_columns(**st.sw_kwargs(), rounding_token=np.zeros((), np.uint32))
    for name in plain_lw._fields:
        np.testing.assert_array_equal(getattr(tok_lw, name), getattr(plain_lw, name))
    for name in plain_sw._fields:
        np.testing.assert_array_equal(getattr(tok_sw, name), getattr(plain_sw, name))
