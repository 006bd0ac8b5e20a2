"""Host-side logic of the Python drop-in that needs no GPU."""

from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize("token", [None, 0, np.uint32(0), np.zeros((3,), np.uint32)])
def test_zero_rounding_tokens_are_accepted(pkg, token):
    from wrf_jax_b200 import rrtmg
    rrtmg._check_rounding_token(token)


@pytest.mark.parametrize("token", [1, np.uint32(0x80000000), np.array([0, 2], np.uint32)])
def test_nonzero_rounding_tokens_are_rejected(pkg, token):
    from wrf_jax_b200 import rrtmg
    with pytest.raises(NotImplementedError):
        rrtmg._check_rounding_token(token)


def test_greenhouse_defaults_follow_the_adapters(pkg):
    from wrf_jax_b200 import rrtmg
    # all five given: used as is (lw:6610-6630)
    assert rrtmg._greenhouse(2020, 1, None, 1e-4, 2e-7, 3e-6, 4e-10, 5e-10, lw=True) == (1e-4, 2e-7, 3e-6, 4e-10, 5e-10)
    # LW with a partial set falls back to the defaults entirely
    co2, n2o, ch4, f11, f12 = rrtmg._greenhouse(2020, 2, None, 1e-4, None, None, None, None, lw=True)
    assert co2 == pytest.approx(379.0e-6) and n2o == pytest.approx(319.0e-9)
    # SW keeps the given scalars and fills the rest (sw:2371-2383)
    sw = rrtmg._greenhouse(2020, 2, None, 1e-4, None, None, None, None, lw=False)
    assert sw[0] == 1e-4 and sw[1] == pytest.approx(319.0e-9) and sw[3:] == (0.0, 0.0)
    # ghg_input == 0: year-dependent CO2
    co2_0 = rrtmg._greenhouse(2000, 0, None, None, None, None, None, None, lw=True)[0]
    assert co2_0 == pytest.approx(370.0e-6)


def test_product_fails_loudly_without_a_gpu(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from wrf_jax_b200 import rrtmg
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        rrtmg.RrtmgContext()


def test_infer_host_rejects_pageable_buffers(pkg):
    """The host-buffer surrogate path reads and writes host memory in place
    from the GPU, so it accepts page-locked tensors only (checked before any
    GPU work)."""
    import torch
    from wrf_jax_b200 import surrogate as S, synthetic
    st = synthetic.make_columns(2, 3, S.NK, seed=1)
    host = {k: torch.from_numpy(v) for k, v in st.fields.items()}
    out = {k: torch.empty((2, S.NK, 3) if k.startswith("rthraten") else (2, 3)) for k in S.OUTPUT_FIELDS}
    with pytest.raises(ValueError):
        S.infer_host(None, st, host, out)


@pytest.mark.parametrize("nx,slabs", [(1000, 8), (425, 8), (9, 8), (3, 8), (2, 8), (1, 8), (100, 3), (100, 2),
                                      (100, 1)])
def test_host_pipeline_slabs_cover_the_rows_once(pkg, nx, slabs):
    from wrf_jax_b200 import surrogate as S
    b = S._slab_bounds(nx, slabs)
    assert b[0][0] == 0 and b[-1][1] == nx
    assert all(i1 > i0 for i0, i1 in b) and all(b[q][1] == b[q + 1][0] for q in range(len(b) - 1))
    assert len(b) <= min(slabs, nx)
    if nx >= 4 * slabs and slabs >= 3:  # the last two slabs taper to a half and a quarter
        sizes = [i1 - i0 for i0, i1 in b]
        assert sizes[-1] < sizes[-2] < sizes[0]
