"""Generate the radiation-tendency golden fixtures from the reference's own code.

Run here (the machine that has the WRF-JAX sources); the GPU box only reads the
committed output:

    python tests/golden/make_tendency_golden.py /path/to/WRF-JAX

The chain after the RRTMG calls, as the reference runs it:

1. ``rthraten = rthratenlw + rthratensw`` (src/wrf_jax/runtime.py:7946, one
   binary32 addition; restated here, it is that one line);
2. ``calculate_phy_tend`` (src/wrf_jax/dyn_em/module_em.py:462) couples it with
   the column mass, rthraten * (c1[k] * mut + c2[k]) over the tile;
3. ``phy_ra_ten`` (src/wrf_jax/physics/module_physics_addtendc.py:542, through
   ``add_a2a``) adds it to the potential-temperature tendency over the tile
   less the specified / nested boundary rows.

Steps 2 and 3 run the reference's functions under ``tests/golden/jaxshim.py``:
module_physics_addtendc imports as it is; module_em imports jax internals, so
``calculate_phy_tend`` (and the ``_read`` helper of module_advect_em, and the
tracer index constants of module_em) are parsed out of their files and run
unchanged.  Every other tendency passed to ``calculate_phy_tend`` is zero and
only the radiation schemes are switched on.

Output: tendency_golden.npz.
"""

from __future__ import annotations

import ast
import os
import sys
from collections.abc import Mapping
from pathlib import Path
from typing import Any

import numpy as np

HERE = Path(__file__).resolve().parent

# name: memory extents (ims..ime, kms..kme, jms..jme), domain (ids..ide, kds..kde, jds..jde),
# tile (its..ite, kts..kte, jts..jte), specified, nested, periodic_x
CASES = (
    ("tile_halo_spec", dict(ims=-2, ime=14, kms=1, kme=31, jms=-2, jme=11, ids=1, ide=13, kds=1, kde=31,
                            jds=1, jde=10, its=1, ite=12, kts=1, kte=30, jts=1, jte=9,
                            specified=True, nested=False, periodic_x=False)),
    ("interior_tile", dict(ims=3, ime=12, kms=1, kme=45, jms=2, jme=9, ids=1, ide=20, kds=1, kde=45,
                           jds=1, jde=15, its=5, ite=10, kts=1, kte=44, jts=4, jte=7,
                           specified=False, nested=False, periodic_x=False)),
    ("periodic_nested", dict(ims=1, ime=9, kms=1, kme=21, jms=1, jme=7, ids=1, ide=9, kds=1, kde=21,
                             jds=1, jde=7, its=1, ite=9, kts=1, kte=21, jts=1, jte=7,
                             specified=False, nested=True, periodic_x=True)),
    ("whole_domain", dict(ims=1, ime=33, kms=1, kme=51, jms=1, jme=17, ids=1, ide=33, kds=1, kde=51,
                          jds=1, jde=17, its=1, ite=33, kts=1, kte=51, jts=1, jte=17,
                          specified=False, nested=False, periodic_x=False)),
)


def extract(path: Path, names: tuple, ns: dict) -> None:
    tree = ast.parse(path.read_text())
    for node in tree.body:
        hit = (isinstance(node, ast.FunctionDef) and node.name in names) or (
            isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id in names for t in node.targets))
        if hit:
            exec(compile(ast.Module(body=[node], type_ignores=[]), str(path), "exec"), ns)


def main(reference_root: str) -> None:
    sys.path.insert(0, str(HERE))
    import jaxshim

    jaxshim.install()
    src = Path(reference_root) / "src"
    sys.path.insert(0, str(src))
    import jax.numpy as jnp
    from jax import lax
    from wrf_jax.physics import module_physics_addtendc as addt

    ns: dict[str, Any] = dict(jnp=jnp, lax=lax, Any=Any, Mapping=Mapping)
    extract(src / "wrf_jax" / "dyn_em" / "module_advect_em.py", ("_read",), ns)
    extract(src / "wrf_jax" / "dyn_em" / "module_em.py",
            ("PARAM_FIRST_SCALAR", "P_QV", "P_QC", "P_QR", "P_QI", "P_QS", "P_QG", "calculate_phy_tend"), ns)
    calc = ns["calculate_phy_tend"]
    import inspect
    params = list(inspect.signature(calc).parameters)

    out = {}
    rng = np.random.default_rng(7)
    for name, b in CASES:
        nx, nk, ny = b["ime"] - b["ims"] + 1, b["kme"] - b["kms"] + 1, b["jme"] - b["jms"] + 1
        lw = rng.normal(-2e-5, 1e-5, (nx, nk, ny)).astype(np.float32)
        sw = np.maximum(rng.normal(1e-5, 1e-5, (nx, nk, ny)), 0).astype(np.float32)
        c1 = rng.uniform(0.0, 1.0, nk).astype(np.float32)
        c2 = rng.uniform(0.0, 5000.0, nk).astype(np.float32)
        mut = rng.uniform(5.0e4, 9.5e4, (nx, ny)).astype(np.float32)
        rt_tendf = rng.normal(0.0, 3.0, (nx, nk, ny)).astype(np.float32)
        rthraten = np.asarray(jnp.asarray(lw, dtype=jnp.float32) + jnp.asarray(sw, dtype=jnp.float32))
        cfg = dict(ra_lw_physics=4, ra_sw_physics=4, specified=b["specified"], nested=b["nested"],
                   periodic_x=b["periodic_x"])
        zero3 = np.zeros((nx, nk, ny), np.float32)
        args = {}
        for pname in params:
            if pname == "config_flags":
                args[pname] = cfg
            elif pname in ("c1", "c2"):
                args[pname] = c1 if pname == "c1" else c2
            elif pname in ("mut", "muu", "muv"):
                args[pname] = mut
            elif pname == "rthraten":
                args[pname] = rthraten
            elif pname in ("num_scalar", "num_tracer"):
                args[pname] = 0
            elif pname in ("scalar", "scalar_tend", "tracer", "tracer_tend"):
                args[pname] = np.zeros((nx, nk, ny, 1), np.float32)
            elif pname in b:
                args[pname] = b[pname]
            elif pname in ("rounding_token", "p_qv", "p_qc", "p_qr", "p_qi", "p_qs", "p_qg",
                           "param_first_scalar"):
                continue
            else:
                args[pname] = zero3
        coupled = np.asarray(calc(**args)[0], np.float32)
        bounds = {k: b[k] for k in ("ids", "ide", "jds", "jde", "kds", "kde", "ims", "ime", "jms", "jme",
                                    "kms", "kme", "its", "ite", "jts", "jte", "kts", "kte")}
        tend = np.asarray(addt.phy_ra_ten(cfg, rt_tendf, coupled, **bounds), np.float32)
        for k, v in dict(lw=lw, sw=sw, c1=c1, c2=c2, mut=mut, rt_tendf=rt_tendf, rthraten=coupled,
                         rt_tendf_out=tend).items():
            out[f"{name}/{k}"] = np.ascontiguousarray(v)
        out[f"{name}/bounds"] = np.asarray(
            [b[k] for k in ("ids", "ide", "jds", "jde", "kds", "kde", "ims", "ime", "jms", "jme", "kms",
                            "kme", "its", "ite", "jts", "jte", "kts", "kte")] +
            [int(b["specified"]), int(b["nested"]), int(b["periodic_x"])], np.int32)
        print("case", name, "done")
    np.savez_compressed(HERE / "tendency_golden.npz", **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
        "WRF_JAX_REFERENCE", str(Path(__file__).resolve().parents[3] / "reference")))
