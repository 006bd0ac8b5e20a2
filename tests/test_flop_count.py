"""The counting build of the oracle (oracle/flop_count.h) and the committed
per-column FP32 operation counts the plain kernels' roofline uses.

* Counting changes no arithmetic: its outputs equal the plain oracle's bit
  for bit.
* tests/golden/flop_counts.json (10 west-east rows of the 425 x 425 x 50
  benchmark domain) agrees with a fresh count on 2 rows of the same domain
  within 2 % (the rows differ in cloud cover and daylight).
"""

from __future__ import annotations

import json

import numpy as np
import pytest

from conftest import GOLDEN, REPO


@pytest.fixture(scope="module")
def counted(blob_path):
    import sys
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as oracle_mod
    return oracle_mod.Oracle(blob_path, counted=True)


def test_counting_changes_no_result(pkg, oracle, counted):
    from wrf_jax_b200 import synthetic
    st = synthetic.make_columns(12, 10, 50, seed=3, fractional_clouds=True)
    for side in ("lwrad", "swrad"):
        kw = st.lw_kwargs() if side == "lwrad" else st.sw_kwargs()
        a, b = getattr(oracle, side)(**kw), getattr(counted, side)(**kw)
        for name in a:
            np.testing.assert_array_equal(np.asarray(a[name]).view(np.uint32), np.asarray(b[name]).view(np.uint32),
                                          err_msg=f"{side} {name}")
    counted.take_counts()


def test_committed_counts_reproduce(pkg, counted):
    import sys
    sys.path.insert(0, str(GOLDEN))
    import make_flop_counts
    ref = json.loads((GOLDEN / "flop_counts.json").read_text())
    fresh = make_flop_counts.count(rows=2)
    for key in ("lw_flops_per_column", "sw_flops_per_day_column"):
        assert abs(fresh[key] / ref[key] - 1.0) < 0.02, (key, fresh[key], ref[key])
    # the division share that makes the SW path more expensive per operation
    assert ref["sw_per_day_column"]["div"] > 0.05 * ref["sw_flops_per_day_column"]
