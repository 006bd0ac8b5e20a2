"""Shared pytest fixtures.

The package directory is ``wrf-jax_b200`` (not an importable name), so it is
loaded by path and registered as ``wrf_jax_b200``.  The oracle under
``oracle/`` is test infrastructure and is only used as the checker here.
"""

from __future__ import annotations

import importlib.util
import os
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
# WRF-JAX sources (only used to build the table blob and the golden fixtures):
# $WRF_JAX_REFERENCE, else a "reference" checkout beside this repository
REFERENCE_ROOT = Path(os.environ.get("WRF_JAX_REFERENCE", str(Path(__file__).resolve().parents[2] / "reference")))
REFERENCE_PHYSICS = REFERENCE_ROOT / "src" / "wrf_jax" / "physics"


def load_package():
    if "wrf_jax_b200" in sys.modules:
        return sys.modules["wrf_jax_b200"]
    root = REPO / "wrf-jax_b200"
    spec = importlib.util.spec_from_file_location(
        "wrf_jax_b200", root / "__init__.py", submodule_search_locations=[str(root)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["wrf_jax_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def blob_path(pkg):
    from wrf_jax_b200 import tables
    if tables.DEFAULT_BLOB.exists():
        return tables.DEFAULT_BLOB
    if REFERENCE_PHYSICS.exists():
        return tables.ensure_blob(REFERENCE_PHYSICS)
    pytest.skip("table blob missing and no WRF-JAX sources to build it from")


@pytest.fixture(scope="session")
def oracle(blob_path):
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle as oracle_mod
    return oracle_mod.Oracle(blob_path, nthreads=os.cpu_count())


@pytest.fixture(scope="session")
def golden():
    with np.load(GOLDEN / "rrtmg_golden.npz") as d:
        data = {k: d[k] for k in d.files}
    cases = {}
    for key, value in data.items():
        case, kind, name = key.split("/")
        cases.setdefault(case, {}).setdefault(kind, {})[name] = value
    return cases


def case_kwargs(case: dict, side: str) -> dict:
    """Rebuild the reference call keywords of one golden case."""
    inp = case["in"]
    common = ("p3d", "p8w", "pi3d", "t3d", "t8w", "tsk", "dz8w", "qv3d", "qc3d", "qi3d",
              "qs3d", "cldfra3d", "o33d", "xland", "xice", "snow", "re_cloud", "re_ice", "re_snow")
    kw = {k: inp[k] for k in common}
    flags = dict(has_reqc=int(inp["has_reqc"]), has_reqi=int(inp["has_reqi"]),
                 has_reqs=int(inp["has_reqs"]), icloud=int(inp["icloud"]),
                 cldovrlp=int(inp["cldovrlp"]), yr=2024, julian=172.5)
    kw.update(flags)
    if side == "lw":
        kw.update(emiss=inp["emiss"], p_top=float(inp["p_top"]),
                  co2vmr=float(inp["co2vmr"]), n2ovmr=float(inp["n2ovmr"]),
                  ch4vmr=float(inp["ch4vmr"]), cfc11vmr=float(inp["cfc11vmr"]),
                  cfc12vmr=float(inp["cfc12vmr"]))
    else:
        kw.update(albedo=inp["albedo"], coszr=inp["coszr"], solcon=float(inp["solcon"]),
                  co2vmr=float(inp["co2vmr"]), n2ovmr=float(inp["n2ovmr"]),
                  ch4vmr=float(inp["ch4vmr"]))
        if "alswvisdir" in inp:  # Noah-MP albedos (sf_surface_physics = 8)
            kw.update(sf_surface_physics=8, **{k: inp[k] for k in ("alswvisdir", "alswvisdif", "alswnirdir",
                                                                    "alswnirdif")})
    return kw
