"""Counted FP32 operations of the plain RRTMG path per column (fixture generator).

Runs the counting build of the oracle (oracle/flop_count.h: every binary32
add/subtract, multiply, divide, sqrt, exp, log and pow the restated reference
path executes) on a sample of the plain benchmark's domain -- the first 10
west-east rows (4,250 columns) of the seeded 425 x 425 x 50 generator domain
(seed 0) -- and writes the averages per LW column and per SW day column to
flop_counts.json beside this script.  bench.py reads that file for the plain
kernels' FP32 roofline; tests/test_flop_count.py checks it against a fresh
count.

    python tests/golden/make_flop_counts.py
"""

from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
OUT = HERE / "flop_counts.json"
SAMPLE_ROWS = 10
WORKLOAD = dict(nx=425, ny=425, nk=50, seed=0)


def sample_kwargs(rows: int = SAMPLE_ROWS):
    sys.path.insert(0, str(REPO / "tests"))
    import conftest

    conftest.load_package()
    from wrf_jax_b200 import synthetic

    st = synthetic.make_columns(WORKLOAD["nx"], WORKLOAD["ny"], WORKLOAD["nk"], seed=WORKLOAD["seed"])

    def cut(kw):
        return {k: (np.ascontiguousarray(v[:rows]) if isinstance(v, np.ndarray) and v.ndim >= 2
                    and v.shape[0] == WORKLOAD["nx"] else v) for k, v in kw.items()}

    return cut(st.lw_kwargs()), cut(st.sw_kwargs())


def count(rows: int = SAMPLE_ROWS) -> dict:
    lw, sw = sample_kwargs(rows)
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle

    from wrf_jax_b200 import tables

    ora = oracle.Oracle(tables.DEFAULT_BLOB, counted=True)
    ora.take_counts()
    ora.lwrad(**lw)
    lw_c = ora.take_counts()
    ora.swrad(**sw)
    sw_c = ora.take_counts()
    ncol = rows * WORKLOAD["ny"]
    nday = int(np.count_nonzero(sw["coszr"] > 0.0))
    return {
        "workload": "plain_%dx%dx%d" % (WORKLOAD["nx"], WORKLOAD["ny"], WORKLOAD["nk"]),
        "sample": f"first {rows} west-east rows ({ncol} columns, {nday} in daylight) of the seed-{WORKLOAD['seed']} domain",
        "counted": "binary32 add/subtract, multiply, divide, sqrt, exp, log, pow executed by the oracle",
        "lw_columns": ncol,
        "sw_day_columns": nday,
        "lw_per_column": {k: v / ncol for k, v in lw_c.items()},
        "sw_per_day_column": {k: v / nday for k, v in sw_c.items()},
        "lw_flops_per_column": sum(lw_c.values()) / ncol,
        "sw_flops_per_day_column": sum(sw_c.values()) / nday,
    }


def main() -> None:
    t = time.time()
    res = count()
    OUT.write_text(json.dumps(res, indent=1) + "\n")
    print(f"wrote {OUT} in {time.time() - t:.1f} s: LW {res['lw_flops_per_column']:.4g} per column, "
          f"SW {res['sw_flops_per_day_column']:.4g} per day column")


if __name__ == "__main__":
    main()
