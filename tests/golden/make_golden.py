"""Generate the golden fixtures from the reference's own RRTMG code.

Run here (the machine that has the WRF-JAX sources); the GPU box only reads the
committed outputs:

    python tests/golden/make_golden.py /path/to/WRF-JAX

WRF-JAX needs jax/jaxlib, which this image does not have, so the reference is
executed under ``tests/golden/jaxshim.py``: a numpy stand-in for the JAX API
surface the RRTMG path touches (jnp/lax operations with JAX's dtype rules,
functional ``.at`` updates, clamped gathers, scan/vmap as loops).  The
reference functions called are the public ones the runtime calls:
``rrtmg_lwrad_wrf_columns`` (module_ra_rrtmg_lw.py:6789) and
``rrtmg_swrad_wrf_columns`` (module_ra_rrtmg_sw.py:2386), plus ``kissvec`` /
``_kiss_random_sequence`` (module_ra_rrtmg_common.py:976, 1067) and the
compressed-table loaders for the table checksums.

Outputs:
  rrtmg_golden.npz    inputs + every LW/SW result field for each case
  kiss_golden.npz     KISS streams for fixed seeds (skip 150 and skip 1)
  tables_sha256.json  sha256 of each compressed absorption table as the
                      reference builds it
"""

from __future__ import annotations

import hashlib
import importlib.util
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]

# Cases: (name, make_columns kwargs, overrides of the call keywords)
CASES = (
    ("c0_4x4x44", dict(nx=4, ny=4, nk=44, seed=0), {}),
    ("c1_3x5x50", dict(nx=3, ny=5, nk=50, seed=1), {}),
    ("req_3x3x44", dict(nx=3, ny=3, nk=44, seed=2, has_req=True), {}),
    ("fraccloud_ptop10_3x3x30", dict(nx=3, ny=3, nk=30, seed=5, fractional_clouds=True,
                                     p_top=1000.0), {}),
    ("allnight_2x3x44", dict(nx=2, ny=3, nk=44, seed=4, night_fraction=1.0), {}),
    ("clearsky_allday_3x2x44", dict(nx=3, ny=2, nk=44, seed=6, cloud_p=0.0,
                                    night_fraction=0.0), {}),
    ("overcast_2x2x40", dict(nx=2, ny=2, nk=40, seed=8, cloud_p=1.0, night_fraction=0.0), {}),
    ("icloud0_2x2x44", dict(nx=2, ny=2, nk=44, seed=3, night_fraction=0.0), dict(icloud=0)),
    ("odd_1x3x17", dict(nx=1, ny=3, nk=17, seed=7, night_fraction=0.0), {}),
    # Noah-MP albedos (sf_surface_physics = 8): half the columns with xland = 2
    # (they keep `albedo`), the others take the four visible / near-infrared
    # fields (module_ra_rrtmg_sw.py:2519-2530)
    ("sf8_3x4x44", dict(nx=3, ny=4, nk=44, seed=9, night_fraction=0.0, fractional_clouds=True), dict(sf8=True)),
)
SF8_FIELDS = ("alswvisdir", "alswvisdif", "alswnirdir", "alswnirdif")


def load_package():
    root = REPO / "wrf-jax_b200"
    spec = importlib.util.spec_from_file_location(
        "wrf_jax_b200", root / "__init__.py", submodule_search_locations=[str(root)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["wrf_jax_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def main(reference_root: str) -> None:
    sys.path.insert(0, str(HERE))
    import jaxshim

    jaxshim.install()
    sys.path.insert(0, str(Path(reference_root) / "src"))
    load_package()
    from wrf_jax_b200 import synthetic
    from wrf_jax.physics import module_ra_rrtmg_common as common
    from wrf_jax.physics import module_ra_rrtmg_lw as lw
    from wrf_jax.physics import module_ra_rrtmg_sw as sw

    out = {}
    for name, gen, over in CASES:
        st = synthetic.make_columns(**gen)
        over = dict(over)
        sf8 = over.pop("sf8", False)
        if sf8:
            rng = np.random.default_rng(99)
            nx, ny = gen["nx"], gen["ny"]
            st.fields["xland"] = np.where(rng.uniform(size=(nx, ny)) < 0.5, 1.0, 2.0).astype(np.float32)
            for k in SF8_FIELDS:
                st.fields[k] = rng.uniform(0.03, 0.5, size=(nx, ny)).astype(np.float32)
        lkw, skw = st.lw_kwargs(), st.sw_kwargs()
        lkw.update(over)
        skw.update(over)
        if sf8:
            skw.update(sf_surface_physics=8, **{k: st.fields[k] for k in SF8_FIELDS})
        for k, v in st.fields.items():
            out[f"{name}/in/{k}"] = v
        for k in ("p_top", "solcon", "co2vmr", "n2ovmr", "ch4vmr", "cfc11vmr", "cfc12vmr",
                  "has_reqc", "has_reqi", "has_reqs"):
            out[f"{name}/in/{k}"] = np.asarray(st.scalars[k])
        out[f"{name}/in/icloud"] = np.asarray(lkw.get("icloud", 1))
        out[f"{name}/in/cldovrlp"] = np.asarray(lkw.get("cldovrlp", 2))
        for k, v in lw.rrtmg_lwrad_wrf_columns(**lkw)._asdict().items():
            out[f"{name}/lw/{k}"] = np.asarray(v, np.float32)
        for k, v in sw.rrtmg_swrad_wrf_columns(**skw)._asdict().items():
            out[f"{name}/sw/{k}"] = np.asarray(v, np.float32)
        print("case", name, "done")
    np.savez_compressed(HERE / "rrtmg_golden.npz", **out)

    # KISS streams: 3 seed sets x 2 skips, 400 draws each.
    seeds = np.asarray([[123456789, 362436069, 521288629, 916191069],
                        [1, 2, 3, 4],
                        [987654321, 5, 77777777, 424242]], np.int32)
    kiss = {"seeds": seeds}
    for skip in (150, 1):
        s = tuple(np.asarray(seeds[:, i]) for i in range(4))
        kiss[f"skip{skip}"] = np.asarray(common._kiss_random_sequence(s, 400, skip), np.float32)
    s1, s2, s3, s4 = (np.asarray(seeds[:, i]) for i in range(4))
    steps = []
    for _ in range(5):
        s1, s2, s3, s4, r = common.kissvec(s1, s2, s3, s4)
        steps.append(np.asarray(r, np.float32))
    kiss["first5"] = np.stack(steps)
    np.savez_compressed(HERE / "kiss_golden.npz", **kiss)

    sha = {}
    L = lw.load_rrtmg_lw_compressed_lookup_tables()
    for b in range(1, 17):
        band = getattr(L, f"band{b}")
        for f in band._fields:
            v = getattr(band, f)
            if f == "band" or v is None:
                continue
            v = np.asarray(v, np.float32)
            if f in ("ka", "kb"):
                v = np.asarray(lw._flatten_ref_table_fortran(v) if v.ndim == 4 else lw._flatten_ref_table_5x(v))
            sha[f"lw{b}.{f}"] = hashlib.sha256(np.ascontiguousarray(v, np.float32).tobytes()).hexdigest()
    S = sw.load_rrtmg_sw_compressed_lookup_tables()
    for b in range(16, 30):
        band = getattr(S, f"band{b}")
        for f in band._fields:
            v = getattr(band, f)
            if f == "band" or v is None:
                continue
            if f in ("ka", "kb"):
                v = np.asarray(v, np.float32)
                v = np.asarray(lw._flatten_ref_table_fortran(v) if v.ndim == 4 else lw._flatten_ref_table_5x(v))
            arr = np.ascontiguousarray(np.asarray(v).reshape(-1) if np.ndim(v) == 0 else np.asarray(v))
            sha[f"sw{b}.{f}"] = hashlib.sha256(arr.tobytes()).hexdigest()
    (HERE / "tables_sha256.json").write_text(json.dumps(sha, indent=1, sort_keys=True) + "\n")
    print("wrote", len(out), "arrays,", len(sha), "table checksums")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
        "WRF_JAX_REFERENCE", str(Path(__file__).resolve().parents[3] / "reference")))
