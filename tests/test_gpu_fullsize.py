"""The CUDA path at full size against the oracle, bit for bit.

Two domains of the seeded generator, every output field of both calls:

* the 425 x 425 x 50 plain-kernel configuration (180,625 columns; the plain
  benchmark's domain, seed 0), which is larger than one LW launch chunk of
  131,072 columns;
* a strip of 200 west-east rows of the 1,000 x 1,000 x 50 surrogate domain
  (seed 2): 200,000 columns, about 140,000 of them in daylight, so the SW day
  list is longer than one launch chunk as well.

The oracle runs on every host core (about 20 s for both domains at the
roughly 18,000 columns/s the C restatement reaches on 16 cores).  Bar:
bit-exact binary32 equality, as for the small domains.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rrtmg(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import rrtmg as mod
    return mod


def _strip(kw: dict, nx: int, rows: int) -> dict:
    out = {}
    for k, v in kw.items():
        if isinstance(v, np.ndarray) and v.ndim >= 2 and v.shape[0] == nx:
            out[k] = np.ascontiguousarray(v[:rows])
        else:
            out[k] = v
    return out


def _compare(rrtmg, oracle, lw_kw: dict, sw_kw: dict, tag: str) -> None:
    for side, call, ref_call, kw in (("lw", rrtmg.rrtmg_lwrad_wrf_columns, oracle.lwrad, lw_kw),
                                     ("sw", rrtmg.rrtmg_swrad_wrf_columns, oracle.swrad, sw_kw)):
        got = call(**kw)._asdict()
        ref = ref_call(**kw)
        for name, value in ref.items():
            g = np.asarray(got[name])
            assert g.shape == value.shape, f"{tag} {side} {name}"
            bad = np.count_nonzero(g.view(np.uint32) != np.asarray(value, np.float32).view(np.uint32))
            assert bad == 0 or np.array_equal(g, value), f"{tag} {side} {name}: {bad} values differ"


def test_config1_425x425x50_matches_oracle(rrtmg, oracle, pkg):
    from wrf_jax_b200 import synthetic
    st = synthetic.make_columns(425, 425, 50, seed=0)
    _compare(rrtmg, oracle, st.lw_kwargs(), st.sw_kwargs(), "425x425x50")


def test_surrogate_domain_strip_matches_oracle(rrtmg, oracle, pkg):
    from wrf_jax_b200 import synthetic
    st = synthetic.make_columns(1000, 1000, 50, seed=2)
    lw, sw = _strip(st.lw_kwargs(), 1000, 200), _strip(st.sw_kwargs(), 1000, 200)
    assert np.count_nonzero(sw["coszr"] > 0) > 131072  # the day list spans two SW launch chunks
    del st
    _compare(rrtmg, oracle, lw, sw, "1000x1000x50 rows 0-199")
