"""Generate the radiation-prologue golden fixtures from the reference's own code.

Run here (the machine that has the WRF-JAX sources); the GPU box only reads the
committed output:

    python tests/golden/make_prologue_golden.py /path/to/WRF-JAX

``src/wrf_jax/runtime.py`` imports jax at module level, which this image does
not have, so the generator parses that file and executes only the host-side
numpy functions the radiation stage calls when its inputs are not traced
(runtime.py:7736-7749): ``_cal_cldfra1_np``, ``_calc_coszen_np`` (with its
SVML and libm helpers), ``_cam_o3rad_np`` (with ``_load_cam_ozone_tables`` and
``_cam_ozone_month_weights``), ``_radconst`` and
``_radiation_greenhouse_scalars``.  Their bodies run unchanged in a namespace
holding numpy, ctypes and pathlib.

The CAM ozone files of a case directory are not shipped with the reference;
a seeded stand-in of the same shape (59 levels x 64 latitudes x 12 months) is
written to a temporary case directory and read back by the reference's loader.

Output: prologue_golden.npz, inputs and outputs per case.
"""

from __future__ import annotations

import ast
import ctypes
import ctypes.util
import importlib.util
import os
import sys
import tempfile
from datetime import datetime
from functools import lru_cache
from pathlib import Path
from typing import Any

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]

FUNCTIONS = ("_radiation_greenhouse_scalars", "_radconst", "_load_cam_ozone_tables",
             "_cam_ozone_month_weights", "_cam_o3rad_np", "_cal_cldfra1_np",
             "_svml_float32_from_bits_np", "_svml_xor_float32_np", "_svml_sinf_np", "_svml_cosf_np",
             "_wrf_scalar_libm", "_wrf_scalar_trig_np", "_calc_coszen_np")

# (name, nx, ny, nk, seed, julian, xtime [min], gmt [h])
CASES = (
    ("summer_7x5x44", 7, 5, 44, 11, 172.3, 3.0 * 60 + 15.0, 6.0),
    ("wrap_dec_4x6x50", 4, 6, 50, 12, 355.2, 1500.0, 18.5),
    ("wrap_jan_9x3x30", 9, 3, 30, 13, 5.4, 20.0, 0.0),
    ("yearend_2x4x44", 2, 4, 44, 14, 364.5, 700.0, 12.0),
    ("spring_13x2x50", 13, 2, 50, 15, 80.0, 4321.0, 23.75),
)


def load_package():
    root = REPO / "wrf-jax_b200"
    spec = importlib.util.spec_from_file_location(
        "wrf_jax_b200", root / "__init__.py", submodule_search_locations=[str(root)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["wrf_jax_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def reference_functions(runtime_py: Path) -> dict:
    tree = ast.parse(runtime_py.read_text())
    ns: dict[str, Any] = dict(np=np, ctypes=ctypes, Path=Path, lru_cache=lru_cache, Any=Any,
                              datetime=datetime, _CAM_OZONE_CACHE={})
    ctypes.util  # noqa: B018 - the libm helper uses ctypes.util through the ctypes module
    found = {}
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name in FUNCTIONS:
            found[node.name] = node
    missing = set(FUNCTIONS) - set(found)
    if missing:
        raise SystemExit(f"reference functions not found: {sorted(missing)}")
    for name in FUNCTIONS:
        code = compile(ast.Module(body=[found[name]], type_ignores=[]), str(runtime_py), "exec")
        exec(code, ns)
    return ns


def edge_fields(st, rng) -> dict:
    """The synthetic column fields plus the branches cal_cldfra1 and the ozone
    interpolation take only at the edges: supersaturated cloudy layers, snow,
    T <= 100 K, p <= 100 Pa, condensate below 1e-12, pressures above the top
    and below the bottom climatology level."""
    f = {k: st.fields[k].copy() for k in ("qv3d", "qc3d", "qi3d", "qs3d", "t3d", "p3d")}
    shape = f["qv3d"].shape
    m = rng.random(shape) < 0.05
    f["qv3d"][m] *= np.float32(1.5)                     # supersaturation -> cldfra 1
    m = rng.random(shape) < 0.15
    f["qs3d"][m] = rng.uniform(0, 3e-4, m.sum()).astype(np.float32)
    m = rng.random(shape) < 0.02
    f["t3d"][m] = np.float32(95.0)
    m = rng.random(shape) < 0.02
    f["p3d"][m] = np.float32(80.0)
    m = rng.random(shape) < 0.03
    f["qc3d"][m] = np.float32(5e-13)
    f["qi3d"][m] = np.float32(0.0)
    f["qs3d"][m] = np.float32(0.0)
    # one column pushed above the climatology's top level (p < 35 Pa)
    f["p3d"][0, :, 0] = np.geomspace(30.0, 2.0, shape[1]).astype(np.float32)
    # and the lowest levels of another below its bottom level (p > 1000 hPa)
    f["p3d"][-1, :2, -1] = np.asarray([101800.0, 100400.0], np.float32)
    return f


def main(reference_root: str) -> None:
    ref = reference_functions(Path(reference_root) / "src" / "wrf_jax" / "runtime.py")
    load_package()
    from wrf_jax_b200 import synthetic

    out = {}
    with tempfile.TemporaryDirectory() as case_dir:
        plev_hpa, lat_oz, ozone = synthetic.cam_ozone_climatology(seed=0)
        synthetic.write_cam_ozone_files(case_dir, plev_hpa, lat_oz, ozone)
        plev, lat_loaded, oz_loaded = ref["_load_cam_ozone_tables"](case_dir)
        out["ozone/plev_pa"] = np.asarray(plev, np.float32)
        out["ozone/lat"] = np.asarray(lat_loaded, np.float32)
        out["ozone/ozone"] = np.asarray(oz_loaded, np.float32)
        for name, nx, ny, nk, seed, julian, xtime, gmt in CASES:
            rng = np.random.default_rng(seed)
            st = synthetic.make_columns(nx=nx, ny=ny, nk=nk, seed=seed, night_fraction=0.0)
            f = edge_fields(st, rng)
            xlat, xlong = synthetic.lat_lon(nx, ny, seed=seed)
            xlat[0, 0], xlat[-1, -1] = np.float32(89.9), np.float32(-89.9)   # beyond the table's latitudes
            declin, solcon = ref["_radconst"](julian)
            prv, nxt, w1, w2 = ref["_cam_ozone_month_weights"](julian)
            pre = f"{name}/"
            for k, v in f.items():
                out[pre + "in/" + k] = v
            out[pre + "in/xlat"] = xlat
            out[pre + "in/xlong"] = xlong
            out[pre + "in/calendar"] = np.asarray([julian, xtime, gmt], np.float64)
            out[pre + "radconst"] = np.asarray([declin, solcon], np.float64)
            out[pre + "month_weights"] = np.asarray([prv, nxt, w1, w2], np.float64)
            for g in (0, 1, 2):
                out[pre + f"ghg{g}"] = np.asarray(
                    ref["_radiation_greenhouse_scalars"](None, 2019, julian, g), np.float32)
            out[pre + "cldfra"] = np.ascontiguousarray(np.asarray(ref["_cal_cldfra1_np"](
                f["qv3d"], f["qc3d"], f["qi3d"], f["qs3d"], f["t3d"], f["p3d"]), np.float32))
            out[pre + "coszen"] = np.ascontiguousarray(np.asarray(ref["_calc_coszen_np"](
                xlat, xlong, julian=julian, xtime=xtime, gmt=gmt, declin=declin), np.float32))
            out[pre + "o33d"] = np.ascontiguousarray(np.asarray(ref["_cam_o3rad_np"](
                xlat, f["p3d"], julian=julian, case_dir=case_dir), np.float32))
            print("case", name, "done")
    np.savez_compressed(HERE / "prologue_golden.npz", **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
        "WRF_JAX_REFERENCE", str(Path(__file__).resolve().parents[3] / "reference")))
