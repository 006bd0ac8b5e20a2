"""Error of the binary32 path and of its FP64 mode against a binary64 run
(test infrastructure; measurement only).

Runs the 425 x 425 x 50 benchmark domain (the seeded generator of
``wrf-jax_b200/synthetic.py``, ``make_columns(425, 425, 50, seed=0)``) through
three builds of the oracle:

* the binary32 restatement (bit for bit the reference, and the GPU's default
  mode);
* the same with ``fp64_steps=1`` (bit for bit the GPU's FP64 mode: SW reftra of
  layers with zwo >= 0.999 or optical depth below 0.1, and the heating rates
  of the five highest model layers in binary64);
* the binary64 build (``fp64.h``: every operation in binary64), standing for
  an FP64 run of the reference path.

For every output field it writes the largest and the root-mean-square
absolute difference of both binary32 modes from the binary64 run (heating
rates converted from K/s of theta to K/day of temperature with pi3d; SW fields
over day columns only) as JSON:

    python oracle/fp64_errors.py [--nx 425 --ny 425 --nk 50] [--out FILE]
"""

from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent


def _package():
    if "wrf_jax_b200" in sys.modules:
        return sys.modules["wrf_jax_b200"]
    root = REPO / "wrf-jax_b200"
    spec = importlib.util.spec_from_file_location(
        "wrf_jax_b200", root / "__init__.py", submodule_search_locations=[str(root)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["wrf_jax_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def field_errors(got: dict, ref: dict, pi3d: np.ndarray, day: np.ndarray | None) -> dict:
    """max / RMS |got - ref| per field; heating in K/day, fluxes in W/m2."""
    out = {}
    for name, r in ref.items():
        if name == "coszr" or name.endswith("cln"):
            continue
        g = np.asarray(got[name], np.float64)
        r = np.asarray(r, np.float64)
        if name.startswith("rthraten"):
            d = (g - r) * pi3d * 86400.0
            if day is not None:
                d = d[np.broadcast_to(day[:, None, :], d.shape)]
            unit = "K/day"
        else:
            d = g - r
            if day is not None:
                d = d[day]
            unit = "W/m2"
        d = np.abs(d)
        out[name] = dict(unit=unit, max=float(d.max()) if d.size else 0.0,
                         rms=float(np.sqrt(np.mean(d * d))) if d.size else 0.0)
    return out


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--nx", type=int, default=425)
    ap.add_argument("--ny", type=int, default=425)
    ap.add_argument("--nk", type=int, default=50)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    _package()
    from wrf_jax_b200 import synthetic, tables

    sys.path.insert(0, str(HERE))
    import oracle

    o32 = oracle.Oracle(tables.DEFAULT_BLOB, nthreads=os.cpu_count())
    o64 = oracle.Oracle(tables.DEFAULT_BLOB, nthreads=os.cpu_count(), binary64=True)
    st = synthetic.make_columns(args.nx, args.ny, args.nk, seed=args.seed)
    result = dict(domain=f"{args.nx}x{args.ny}x{args.nk}", seed=args.seed, columns=args.nx * args.ny)
    t0 = time.time()
    for side in ("lw", "sw"):
        kw = st.lw_kwargs() if side == "lw" else st.sw_kwargs()
        run = (lambda o, **k: o.lwrad(**k)) if side == "lw" else (lambda o, **k: o.swrad(**k))
        ref = run(o64, **kw)
        b32 = run(o32, **kw)
        f64 = run(o32, fp64_steps=1, **kw)
        pi3d = np.asarray(kw["pi3d"], np.float64)
        day = np.asarray(kw["coszr"]) > 0 if side == "sw" else None
        result[side] = dict(binary32=field_errors(b32, ref, pi3d, day),
                            fp64_mode=field_errors(f64, ref, pi3d, day))
        if day is not None:
            result["sw_day_columns"] = int(day.sum())
    result["seconds"] = round(time.time() - t0, 1)
    text = json.dumps(result, indent=1)
    if args.out:
        Path(args.out).write_text(text + "\n")
    print(text)


if __name__ == "__main__":
    main()
