"""Radiation tendency chain (LW + SW heating, mass coupling, accumulation into
the potential-temperature tendency): the oracle against the reference's golden
fixtures on the CPU, and the fused CUDA kernel bit for bit on the GPU."""

from __future__ import annotations

import ctypes
import sys

import numpy as np
import pytest

from conftest import GOLDEN, REPO


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLDEN / "tendency_golden.npz") as d:
        data = {k: d[k] for k in d.files}
    cases = {}
    for key, v in data.items():
        name, field = key.split("/")
        cases.setdefault(name, {})[field] = v
    return cases


@pytest.fixture(scope="module")
def to():
    sys.path.insert(0, str(REPO / "oracle"))
    import tendency_oracle
    return tendency_oracle


def _bounds(c, to):
    bv = c["bounds"]
    b = dict(zip(to.BOUND_NAMES, map(int, bv[:18])))
    b.update(specified=bool(bv[18]), nested=bool(bv[19]), periodic_x=bool(bv[20]))
    return b


def test_oracle_matches_reference_golden(gold, to):
    for name, c in gold.items():
        r, t = to.radiation_tendency(c["lw"], c["sw"], c["c1"], c["c2"], c["mut"], c["rt_tendf"], _bounds(c, to))
        assert np.array_equal(r.view(np.uint32), c["rthraten"].view(np.uint32)), name
        assert np.array_equal(t.view(np.uint32), c["rt_tendf_out"].view(np.uint32)), name


def test_golden_cases_cover_the_regions(gold):
    # coupling and accumulation regions differ (boundary rows) and both leave
    # part of the memory array untouched
    for name, c in gold.items():
        coupled = c["rthraten"] != (c["lw"] + c["sw"])
        added = c["rt_tendf_out"] != c["rt_tendf"]
        assert coupled.any() and added.any() and not added.all(), name
    assert any((c["rthraten"] != c["lw"] + c["sw"]).sum() > (c["rt_tendf_out"] != c["rt_tendf"]).sum()
               for c in gold.values())


def test_c_abi_rejects_bad_arguments_without_gpu(pkg):
    from wrf_jax_b200 import _capi
    lib = _capi.load()
    tb = _capi.TendencyBounds(ids=1, ide=5, jds=1, jde=5, kds=1, kde=5, ims=3, ime=1, jms=1, jme=5, kms=1, kme=5,
                              its=1, ite=5, jts=1, jte=5, kts=1, kte=5)
    p = ctypes.c_void_p(16)
    # ime < ims, missing outputs, coupling without its arrays: rejected before any CUDA call
    assert lib.rrtmg_radiation_tendency(ctypes.byref(tb), p, p, p, p, p, 1, p, p, None) == 1
    tb.ime = 5
    assert lib.rrtmg_radiation_tendency(ctypes.byref(tb), p, p, p, p, p, 1, None, None, None) == 1
    assert lib.rrtmg_radiation_tendency(ctypes.byref(tb), p, p, None, p, p, 1, p, p, None) == 1
    assert lib.rrtmg_phy_ra_ten(ctypes.byref(tb), None, p, None) == 1


@pytest.mark.gpu
def test_gpu_matches_reference_golden(pkg, gold, to):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import tendency
    for name, c in gold.items():
        b = _bounds(c, to)
        flags = {k: b.pop(k) for k in ("specified", "nested", "periodic_x")}
        r, t = tendency.radiation_tendency(c["lw"], c["sw"], c["c1"], c["c2"], c["mut"], c["rt_tendf"], flags, **b)
        np.testing.assert_array_equal(r.view(np.uint32), c["rthraten"].view(np.uint32), err_msg=name)
        np.testing.assert_array_equal(t.view(np.uint32), c["rt_tendf_out"].view(np.uint32), err_msg=name)
        t2 = tendency.phy_ra_ten(flags, c["rt_tendf"], c["rthraten"], **b)
        np.testing.assert_array_equal(t2.view(np.uint32), c["rt_tendf_out"].view(np.uint32), err_msg=name)


@pytest.mark.gpu
@pytest.mark.parametrize("jme", [1205, 1207])  # 1,210 (scalar path) and 1,212 (four per thread) south-north
def test_gpu_matches_oracle_large(pkg, to, jme):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import tendency
    rng = np.random.default_rng(3)
    b = dict(ids=1, ide=301, jds=1, jde=1201, kds=1, kde=51, ims=-4, ime=305, jms=-4, jme=jme, kms=1, kme=51,
             its=1, ite=300, jts=1, jte=1200, kts=1, kte=50)
    shape = (b["ime"] - b["ims"] + 1, b["kme"] - b["kms"] + 1, b["jme"] - b["jms"] + 1)
    lw = rng.normal(-2e-5, 1e-5, shape).astype(np.float32)
    sw = rng.normal(1e-5, 1e-5, shape).astype(np.float32)
    c1 = rng.uniform(0, 1, shape[1]).astype(np.float32)
    c2 = rng.uniform(0, 5000, shape[1]).astype(np.float32)
    mut = rng.uniform(5e4, 9.5e4, (shape[0], shape[2])).astype(np.float32)
    t0 = rng.normal(0, 3, shape).astype(np.float32)
    for flags in (dict(specified=True, nested=False, periodic_x=False),
                  dict(specified=False, nested=False, periodic_x=True)):
        want_r, want_t = to.radiation_tendency(lw, sw, c1, c2, mut, t0, {**b, **flags})
        r, t = tendency.radiation_tendency(lw, sw, c1, c2, mut, t0, flags, **b)
        assert np.array_equal(r.view(np.uint32), want_r.view(np.uint32))
        assert np.array_equal(t.view(np.uint32), want_t.view(np.uint32))
