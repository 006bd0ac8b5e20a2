"""Per-column status of the last call (rrtmg_last_column_errors): clean
columns read 0; a NaN input, a pressure inversion, a temperature outside the
tables and a cloud fraction above 1 set their bits in exactly the columns that
carry them."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import rrtmg, synthetic
    ctx = rrtmg.RrtmgContext()
    ctx.column_status(True)
    yield rrtmg, synthetic, ctx
    ctx.column_status(False)
    ctx.close()


def test_clean_domain_has_no_status_bits(setup):
    rrtmg, synthetic, ctx = setup
    st = synthetic.make_columns(12, 10, 50, seed=3)
    rrtmg.rrtmg_lwrad_wrf_columns(context=ctx, **st.lw_kwargs())
    assert int(ctx.last_column_errors("lw", 12, 10).abs().sum()) == 0
    rrtmg.rrtmg_swrad_wrf_columns(context=ctx, **st.sw_kwargs())
    assert int(ctx.last_column_errors("sw", 12, 10).abs().sum()) == 0


def test_bad_columns_are_flagged(setup):
    rrtmg, synthetic, ctx = setup
    st = synthetic.make_columns(12, 10, 50, seed=4, night_fraction=0.0)
    f = st.fields
    f["qv3d"][1, 7, 2] = np.nan                       # column (1, 2): NaN input
    f["p8w"][3, 20, 4] = f["p8w"][3, 19, 4] + 10.0   # column (3, 4): pressure inversion
    f["t3d"][5, 30, 6] = 350.0                       # column (5, 6): beyond the Planck table
    f["cldfra3d"][7, 3, 8] = 1.5                     # column (7, 8): cloud fraction above 1
    want = np.zeros((12, 10), np.int64)
    want[1, 2] |= ctx.COL_NONFINITE_INPUT
    want[3, 4] |= ctx.COL_PRESSURE_ORDER
    want[5, 6] |= ctx.COL_TEMPERATURE_RANGE
    want[7, 8] |= ctx.COL_FRACTION_RANGE
    for side, fn, kw in (("lw", rrtmg.rrtmg_lwrad_wrf_columns, st.lw_kwargs()),
                         ("sw", rrtmg.rrtmg_swrad_wrf_columns, st.sw_kwargs())):
        res = fn(context=ctx, **kw)
        got = ctx.last_column_errors(side, 12, 10).cpu().numpy().astype(np.int64)
        nonfinite_out = ~np.isfinite(np.asarray(getattr(res, "rthratenlw" if side == "lw" else "rthratensw"))).all(axis=1)
        exp = want.copy()
        exp[nonfinite_out] |= ctx.COL_NONFINITE_OUTPUT
        np.testing.assert_array_equal(got, exp, err_msg=side)


def test_status_requires_a_recorded_call(setup):
    rrtmg, _, ctx = setup
    with pytest.raises(rrtmg.RrtmgError):
        ctx.last_column_errors("lw", 1, 7)
