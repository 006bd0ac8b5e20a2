"""Build the RRTMG table blob consumed by ``librrtmg_b200.so`` (and the oracle).

Sources, all read from a WRF-JAX installation (``src/wrf_jax/physics``):

* ``data/rrtmg/RRTMG_LW_DATA`` and ``RRTMG_SW_DATA``: big-endian Fortran
  unformatted records, one per band, fields in Fortran order.  The record
  layouts are the ones WRF's ``rrtmg_lw_read_nc``/``rrtmg_sw_read_nc`` use
  (reference: ``module_ra_rrtmg_lw.py:588-782``, ``module_ra_rrtmg_sw.py:844-1014``).
* ``data/rrtmg_{lw,sw}_{cloud,pade,setcoef}_tables.npz``: cloud optics, the
  exact WRF Pade tables and the LW reference atmosphere / Planck tables.
* literal tables in the Python sources (ice radius table, ozone climatology,
  LW buffer-layer standard profile, SW reference atmosphere, g-point maps),
  read with :mod:`ast` so no reference code is executed.

The 256 -> 140 (LW) and 224 -> 112 (SW) g-point reduction (WRF ``cmbgb*``) is
restated here: ``rwgt`` is built in binary32 exactly as WRF initialises it
(``module_ra_rrtmg_common.py:650-689``) and each compressed coefficient is the
binary32 running sum, in original g-point order, of ``raw * rwgt`` (or of the
raw values for Planck fractions and solar source functions;
``module_ra_rrtmg_lw.py:829-910``, ``module_ra_rrtmg_sw.py:1068-1130``).

Blob layout (little endian): ``b"RRTMGB2\\0"``, u32 version, u32 count, then
``count`` entries of {char name[48]; u32 dtype (0=f32, 1=i32, 2=f64, 3=u64); u32 ndim;
u32 shape[4]; u64 offset; u64 nbytes}, then the data, each array 256-byte
aligned.  Absorption tables ``ka``/``kb`` are stored as 2-D
``(rows, ngc)`` with row = ``(jp * n_t + jt) * n_species + js`` (the Fortran
``absa(ind, ig)`` flattening; ``module_ra_rrtmg_lw.py:1444-1452``).
"""

from __future__ import annotations

import ast
import struct
from pathlib import Path

import numpy as np

MAGIC = b"RRTMGB2\0"
VERSION = 1
MG = 16


# ---------------------------------------------------------------------------
# literal tables from the reference sources
# ---------------------------------------------------------------------------
def _literal_tables(path: Path, names: tuple[str, ...]) -> dict:
    tree = ast.parse(path.read_text())
    found = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and len(node.targets) == 1 and isinstance(node.targets[0], ast.Name):
            name = node.targets[0].id
            if name in names:
                value = node.value
                if isinstance(value, ast.Call):  # jnp.asarray((...), dtype=...)
                    value = value.args[0]
                found[name] = ast.literal_eval(value)
    missing = set(names) - set(found)
    if missing:
        raise ValueError(f"literal tables not found in {path}: {sorted(missing)}")
    return found


def _hex_floats(node) -> list:
    """All float.fromhex("...") literals under an AST node, in source order."""
    vals = []
    for sub in ast.walk(node):
        if (isinstance(sub, ast.Call) and isinstance(sub.func, ast.Attribute)
                and sub.func.attr == "fromhex" and sub.args
                and isinstance(sub.args[0], ast.Constant)):
            vals.append((sub.lineno, sub.col_offset, float.fromhex(sub.args[0].value)))
    return [v for _, _, v in sorted(vals)]


def _glibc_math_tables(path: Path) -> dict:
    """glibc 2.39 logf/expf data as the reference reproduces it (core/wrf_math.py).

    These are glibc's published constants (sysdeps/ieee754/flt-32/e_logf_data.c,
    e_exp2f_data.c): 16 (1/c, log c) pairs and a cubic for logf; 32 table
    entries of 2^(i/32) bit patterns, the scaled 1/ln2 and a cubic for expf.
    """
    tree = ast.parse(path.read_text())
    nodes = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and len(node.targets) == 1 and isinstance(node.targets[0], ast.Name):
            nodes[node.targets[0].id] = node.value
    logf_tab = np.asarray(_hex_floats(nodes["_GLIBC_LOGF_TABLE_NP"]), np.float64).reshape(16, 2)
    ln2 = _hex_floats(nodes["_GLIBC_LOGF_LN2"])
    logf_poly = np.asarray(_hex_floats(nodes["_GLIBC_LOGF_POLY"]), np.float64)
    exp_ints = [int(sub.value) for sub in ast.walk(nodes["_GLIBC_EXPF_TABLE"])
                if isinstance(sub, ast.Constant) and isinstance(sub.value, int) and sub.value > 2**32]
    inv_ln2 = _hex_floats(nodes["_GLIBC_EXPF_INV_LN2_SCALED"])
    exp_poly = np.asarray(_hex_floats(nodes["_GLIBC_EXPF_POLY"]), np.float64)
    if logf_tab.shape != (16, 2) or len(ln2) != 1 or logf_poly.size != 3:
        raise ValueError("unexpected glibc logf data layout")
    if len(exp_ints) != 32 or len(inv_ln2) != 1 or exp_poly.size != 3:
        raise ValueError("unexpected glibc expf data layout")
    return {
        "glibc.logf_invc_logc": np.ascontiguousarray(logf_tab),
        "glibc.logf_ln2_poly": np.asarray([ln2[0], *logf_poly], np.float64),
        "glibc.expf_tab": np.asarray(exp_ints, np.uint64),
        "glibc.expf_invln2n_poly": np.asarray([inv_ln2[0], *exp_poly], np.float64),
    }



def _svml_trig_constants(runtime_py: Path) -> dict:
    """Constants of the four-lane SVML sin/cos emulation the zenith-angle code
    uses (src/wrf_jax/runtime.py, ``_svml_sinf_np`` / ``_svml_cosf_np``): the
    bit patterns passed to ``_svml_float32_from_bits_np`` in source order,
    stored as binary32 (12 for sin, 14 for cos)."""
    tree = ast.parse(runtime_py.read_text())
    out = {}
    for fname, key, count in (("_svml_sinf_np", "svml.sinf", 12), ("_svml_cosf_np", "svml.cosf", 14)):
        node = next((n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == fname), None)
        if node is None:
            raise ValueError(f"{runtime_py}: {fname} not found")
        calls = sorted(
            (sub.lineno, sub.col_offset, int(sub.args[0].value)) for sub in ast.walk(node)
            if isinstance(sub, ast.Call) and isinstance(sub.func, ast.Name)
            and sub.func.id == "_svml_float32_from_bits_np" and sub.args
            and isinstance(sub.args[0], ast.Constant))
        bits = [b for _, _, b in calls]
        if len(bits) != count:
            raise ValueError(f"{fname}: expected {count} constants, found {len(bits)}")
        out[key] = np.asarray(bits, np.uint32).view(np.float32).copy()
    return out

# ---------------------------------------------------------------------------
# Fortran record parsing
# ---------------------------------------------------------------------------
_LW_RECORDS = {
    1: (("fracrefao", "r", (16,)), ("fracrefbo", "r", (16,)), ("kao", "r", (5, 13, 16)),
        ("kbo", "r", (5, 47, 16)), ("kao_mn2", "r", (19, 16)), ("kbo_mn2", "r", (19, 16)),
        ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    2: (("fracrefao", "r", (16,)), ("fracrefbo", "r", (16,)), ("kao", "r", (5, 13, 16)),
        ("kbo", "r", (5, 47, 16)), ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    3: (("fracrefao", "r", (16, 9)), ("fracrefbo", "r", (16, 5)), ("kao", "r", (9, 5, 13, 16)),
        ("kbo", "r", (5, 5, 47, 16)), ("kao_mn2o", "r", (9, 19, 16)), ("kbo_mn2o", "r", (5, 19, 16)),
        ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    4: (("fracrefao", "r", (16, 9)), ("fracrefbo", "r", (16, 5)), ("kao", "r", (9, 5, 13, 16)),
        ("kbo", "r", (5, 5, 47, 16)), ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    5: (("fracrefao", "r", (16, 9)), ("fracrefbo", "r", (16, 5)), ("kao", "r", (9, 5, 13, 16)),
        ("kbo", "r", (5, 5, 47, 16)), ("kao_mo3", "r", (9, 19, 16)), ("ccl4o", "r", (16,)),
        ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    6: (("fracrefao", "r", (16,)), ("kao", "r", (5, 13, 16)), ("kao_mco2", "r", (19, 16)),
        ("cfc11adjo", "r", (16,)), ("cfc12o", "r", (16,)), ("selfrefo", "r", (10, 16)),
        ("forrefo", "r", (4, 16))),
    7: (("fracrefao", "r", (16, 9)), ("fracrefbo", "r", (16,)), ("kao", "r", (9, 5, 13, 16)),
        ("kbo", "r", (5, 47, 16)), ("kao_mco2", "r", (9, 19, 16)), ("kbo_mco2", "r", (19, 16)),
        ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    8: (("fracrefao", "r", (16,)), ("fracrefbo", "r", (16,)), ("kao", "r", (5, 13, 16)),
        ("kbo", "r", (5, 47, 16)), ("kao_mco2", "r", (19, 16)), ("kbo_mco2", "r", (19, 16)),
        ("kao_mn2o", "r", (19, 16)), ("kbo_mn2o", "r", (19, 16)), ("kao_mo3", "r", (19, 16)),
        ("cfc12o", "r", (16,)), ("cfc22adjo", "r", (16,)), ("selfrefo", "r", (10, 16)),
        ("forrefo", "r", (4, 16))),
    9: (("fracrefao", "r", (16, 9)), ("fracrefbo", "r", (16,)), ("kao", "r", (9, 5, 13, 16)),
        ("kbo", "r", (5, 47, 16)), ("kao_mn2o", "r", (9, 19, 16)), ("kbo_mn2o", "r", (19, 16)),
        ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    10: (("fracrefao", "r", (16,)), ("fracrefbo", "r", (16,)), ("kao", "r", (5, 13, 16)),
         ("kbo", "r", (5, 47, 16)), ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    11: (("fracrefao", "r", (16,)), ("fracrefbo", "r", (16,)), ("kao", "r", (5, 13, 16)),
         ("kbo", "r", (5, 47, 16)), ("kao_mo2", "r", (19, 16)), ("kbo_mo2", "r", (19, 16)),
         ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    12: (("fracrefao", "r", (16, 9)), ("kao", "r", (9, 5, 13, 16)), ("selfrefo", "r", (10, 16)),
         ("forrefo", "r", (4, 16))),
    13: (("fracrefao", "r", (16, 9)), ("fracrefbo", "r", (16,)), ("kao", "r", (9, 5, 13, 16)),
         ("kao_mco2", "r", (9, 19, 16)), ("kao_mco", "r", (9, 19, 16)), ("kbo_mo3", "r", (19, 16)),
         ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    14: (("fracrefao", "r", (16,)), ("fracrefbo", "r", (16,)), ("kao", "r", (5, 13, 16)),
         ("kbo", "r", (5, 47, 16)), ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    15: (("fracrefao", "r", (16, 9)), ("kao", "r", (9, 5, 13, 16)), ("kao_mn2", "r", (9, 19, 16)),
         ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
    16: (("fracrefao", "r", (16, 9)), ("fracrefbo", "r", (16,)), ("kao", "r", (9, 5, 13, 16)),
         ("kbo", "r", (5, 47, 16)), ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16))),
}

_SW_RECORDS = {
    16: (("rayl", "r", None), ("strrat1", "r", None), ("layreffr", "i", None),
         ("kao", "r", (9, 5, 13, 16)), ("kbo", "r", (5, 47, 16)), ("selfrefo", "r", (10, 16)),
         ("forrefo", "r", (3, 16)), ("sfluxrefo", "r", (16,))),
    17: (("rayl", "r", None), ("strrat", "r", None), ("layreffr", "i", None),
         ("kao", "r", (9, 5, 13, 16)), ("kbo", "r", (5, 5, 47, 16)), ("selfrefo", "r", (10, 16)),
         ("forrefo", "r", (4, 16)), ("sfluxrefo", "r", (16, 5))),
    18: (("rayl", "r", None), ("strrat", "r", None), ("layreffr", "i", None),
         ("kao", "r", (9, 5, 13, 16)), ("kbo", "r", (5, 47, 16)), ("selfrefo", "r", (10, 16)),
         ("forrefo", "r", (3, 16)), ("sfluxrefo", "r", (16, 9))),
    19: (("rayl", "r", None), ("strrat", "r", None), ("layreffr", "i", None),
         ("kao", "r", (9, 5, 13, 16)), ("kbo", "r", (5, 47, 16)), ("selfrefo", "r", (10, 16)),
         ("forrefo", "r", (3, 16)), ("sfluxrefo", "r", (16, 9))),
    20: (("rayl", "r", None), ("layreffr", "i", None), ("absch4o", "r", (16,)),
         ("kao", "r", (5, 13, 16)), ("kbo", "r", (5, 47, 16)), ("selfrefo", "r", (10, 16)),
         ("forrefo", "r", (4, 16)), ("sfluxrefo", "r", (16,))),
    21: (("rayl", "r", None), ("strrat", "r", None), ("layreffr", "i", None),
         ("kao", "r", (9, 5, 13, 16)), ("kbo", "r", (5, 5, 47, 16)), ("selfrefo", "r", (10, 16)),
         ("forrefo", "r", (4, 16)), ("sfluxrefo", "r", (16, 9))),
    22: (("rayl", "r", None), ("strrat", "r", None), ("layreffr", "i", None),
         ("kao", "r", (9, 5, 13, 16)), ("kbo", "r", (5, 47, 16)), ("selfrefo", "r", (10, 16)),
         ("forrefo", "r", (3, 16)), ("sfluxrefo", "r", (16, 9))),
    23: (("raylo", "r", (16,)), ("givfac", "r", None), ("layreffr", "i", None),
         ("kao", "r", (5, 13, 16)), ("selfrefo", "r", (10, 16)), ("forrefo", "r", (3, 16)),
         ("sfluxrefo", "r", (16,))),
    24: (("raylao", "r", (16, 9)), ("raylbo", "r", (16,)), ("strrat", "r", None),
         ("layreffr", "i", None), ("abso3ao", "r", (16,)), ("abso3bo", "r", (16,)),
         ("kao", "r", (9, 5, 13, 16)), ("kbo", "r", (5, 47, 16)), ("selfrefo", "r", (10, 16)),
         ("forrefo", "r", (3, 16)), ("sfluxrefo", "r", (16, 9))),
    25: (("raylo", "r", (16,)), ("layreffr", "i", None), ("abso3ao", "r", (16,)),
         ("abso3bo", "r", (16,)), ("kao", "r", (5, 13, 16)), ("sfluxrefo", "r", (16,))),
    26: (("raylo", "r", (16,)), ("sfluxrefo", "r", (16,))),
    27: (("raylo", "r", (16,)), ("scalekur", "r", None), ("layreffr", "i", None),
         ("kao", "r", (5, 13, 16)), ("kbo", "r", (5, 47, 16)), ("sfluxrefo", "r", (16,))),
    28: (("rayl", "r", None), ("strrat", "r", None), ("layreffr", "i", None),
         ("kao", "r", (9, 5, 13, 16)), ("kbo", "r", (5, 5, 47, 16)), ("sfluxrefo", "r", (16, 5))),
    29: (("rayl", "r", None), ("layreffr", "i", None), ("absh2oo", "r", (16,)),
         ("absco2o", "r", (16,)), ("kao", "r", (5, 13, 16)), ("kbo", "r", (5, 47, 16)),
         ("selfrefo", "r", (10, 16)), ("forrefo", "r", (4, 16)), ("sfluxrefo", "r", (16,))),
}


def _read_records(path: Path, layouts: dict) -> dict:
    raw = path.read_bytes()
    pos = 0
    out = {}
    for band, fields in layouts.items():
        (n,) = struct.unpack_from(">i", raw, pos)
        body = raw[pos + 4: pos + 4 + n]
        (n2,) = struct.unpack_from(">i", raw, pos + 4 + n)
        if n2 != n:
            raise ValueError(f"{path}: record markers differ for band {band}")
        pos += 8 + n
        off = 0
        values = {}
        for name, kind, shape in fields:
            count = 1 if shape is None else int(np.prod(shape))
            dt = np.dtype(">f4" if kind == "r" else ">i4")
            arr = np.frombuffer(body, dtype=dt, count=count, offset=off)
            off += count * 4
            if shape is None:
                values[name] = arr.astype(np.float32 if kind == "r" else np.int32)[0]
            else:
                values[name] = np.array(arr.reshape(shape, order="F"),
                                        dtype=np.float32 if kind == "r" else np.int32)
        if off != len(body):
            raise ValueError(f"{path}: band {band} record has {len(body) - off} extra bytes")
        out[band] = values
    if pos != len(raw):
        raise ValueError(f"{path}: {len(raw) - pos} trailing bytes")
    return out


# ---------------------------------------------------------------------------
# g-point reduction
# ---------------------------------------------------------------------------
def _rwgt(ngc, ngm, ngn, wt) -> np.ndarray:
    """binary32 reduction weights, WRF ``rrtmg_*_init`` order."""
    wt32 = [np.float32(w) for w in wt]
    nband = len(ngc)
    rwgt = np.zeros(nband * MG, np.float32)
    igcsm = 0
    for ib in range(nband):
        if ngc[ib] < MG:
            wtsm = np.zeros(ngc[ib], np.float32)
            iprsm = 0
            for igc in range(ngc[ib]):
                s = np.float32(0.0)
                for _ in range(ngn[igcsm]):
                    s = np.float32(s + wt32[iprsm])
                    iprsm += 1
                igcsm += 1
                wtsm[igc] = s
            for ig in range(MG):
                ind = ib * MG + ig
                rwgt[ind] = np.float32(wt32[ig] / wtsm[ngm[ind] - 1])
        else:
            igcsm += ngc[ib]
            rwgt[ib * MG: (ib + 1) * MG] = np.float32(1.0)
    return rwgt


def _groups(ib, ngc, ngs, ngn, rwgt):
    start = 0 if ib == 0 else ngs[ib - 1]
    pos = 0
    groups = []
    for igc in range(ngc[ib]):
        cnt = ngn[start + igc]
        groups.append((pos, pos + cnt, rwgt[ib * MG + pos: ib * MG + pos + cnt]))
        pos += cnt
    assert pos == MG
    return groups


def _reduce(arr, groups, axis, weighted):
    """Sequential binary32 sums of (weighted) original g-points along ``axis``."""
    arr = np.moveaxis(np.asarray(arr, np.float32), axis, -1)
    out = np.empty(arr.shape[:-1] + (len(groups),), np.float32)
    for igc, (a, b, w) in enumerate(groups):
        acc = np.zeros(arr.shape[:-1], np.float32)
        for k in range(a, b):
            term = (arr[..., k] * w[k - a]).astype(np.float32) if weighted else arr[..., k]
            acc = (acc + term).astype(np.float32)
        out[..., igc] = acc
    return np.moveaxis(out, -1, axis)


def _flatten_rows(k: np.ndarray) -> np.ndarray:
    """(js, jt, jp, g) or (jt, jp, g) -> (rows, g), row = (jp*nt + jt)*ns + js."""
    if k.ndim == 3:
        k = k[None]
    ns, nt, npr, ng = k.shape
    return np.ascontiguousarray(np.transpose(k, (2, 1, 0, 3)).reshape(npr * nt * ns, ng))


def _compress(raw: dict, ib, ngc, ngs, ngn, rwgt, prefix: str) -> dict:
    groups = _groups(ib, ngc, ngs, ngn, rwgt)
    out = {}
    for name, value in raw.items():
        if isinstance(value, (np.floating, np.integer)) or np.ndim(value) == 0:
            out[f"{prefix}.{name}"] = np.asarray(value).reshape(1)
            continue
        if name.startswith(("kao_", "kbo_")):
            base = name[:2] + name[3:]
        elif name.endswith("o") and name != "raylo":
            base = name[:-1]
        else:
            base = name
        if name in ("fracrefao", "fracrefbo", "sfluxrefo"):
            red = _reduce(value, groups, 0, weighted=False)          # (ngc, ...)
            out[f"{prefix}.{base}"] = np.ascontiguousarray(red)
        elif name in ("ccl4o", "cfc11adjo", "cfc12o", "cfc22adjo", "absch4o", "abso3ao",
                      "abso3bo", "absh2oo", "absco2o", "raylo", "raylao", "raylbo"):
            red = _reduce(value, groups, 0, weighted=True)
            key = "rayl" if name == "raylo" else base
            out[f"{prefix}.{key}"] = np.ascontiguousarray(red)
        elif name in ("kao", "kbo"):
            red = _reduce(value, groups, value.ndim - 1, weighted=True)
            out[f"{prefix}.{base}"] = _flatten_rows(red)
        else:  # minor / continuum tables, g-point last
            red = _reduce(value, groups, value.ndim - 1, weighted=True)
            out[f"{prefix}.{base}"] = np.ascontiguousarray(red)
    return out


# ---------------------------------------------------------------------------
# assemble
# ---------------------------------------------------------------------------
def build_tables(physics_dir: str | Path) -> dict:
    """Return {name: ndarray} for every table the radiation path reads."""
    phys = Path(physics_dir)
    data = phys / "data"
    common = _literal_tables(phys / "module_ra_rrtmg_common.py", (
        "RETAB", "_O3SUM", "_PPSUM", "_O3WIN", "_PPWIN", "_RRTMG_WT_VALUES",
        "_LW_GPOINT_COUNTS", "_SW_GPOINT_COUNTS", "_LW_NGS_VALUES", "_LW_NGM_VALUES",
        "_LW_NGN_VALUES", "_SW_NGS_VALUES", "_SW_NGM_VALUES", "_SW_NGN_VALUES"))
    lwlit = _literal_tables(phys / "module_ra_rrtmg_lw.py", ("_LW_BUFFER_PPROF", "_LW_BUFFER_TPROF"))
    swlit = _literal_tables(phys / "module_ra_rrtmg_sw.py", ("_PREFLOG_VALUES", "_TREF_VALUES"))

    t: dict[str, np.ndarray] = {}
    f32 = lambda x: np.ascontiguousarray(np.asarray(x, np.float32))
    i32 = lambda x: np.ascontiguousarray(np.asarray(x, np.int32))

    t["retab"] = f32(common["RETAB"])
    t["o3sum"] = f32(common["_O3SUM"])
    t["ppsum"] = f32(common["_PPSUM"])
    t["o3win"] = f32(common["_O3WIN"])
    t["ppwin"] = f32(common["_PPWIN"])
    t["lw_buffer_pprof"] = f32(lwlit["_LW_BUFFER_PPROF"])
    t["lw_buffer_tprof"] = f32(lwlit["_LW_BUFFER_TPROF"])
    t["sw.preflog"] = f32(swlit["_PREFLOG_VALUES"])
    t.update(_glibc_math_tables(phys.parent / "core" / "wrf_math.py"))
    t.update(_svml_trig_constants(phys.parent / "runtime.py"))
    t["sw.tref"] = f32(swlit["_TREF_VALUES"])

    for side, counts, ngs, ngm, ngn, nb, first, records, fname in (
        ("lw", common["_LW_GPOINT_COUNTS"], common["_LW_NGS_VALUES"], common["_LW_NGM_VALUES"],
         common["_LW_NGN_VALUES"], 16, 1, _LW_RECORDS, "RRTMG_LW_DATA"),
        ("sw", common["_SW_GPOINT_COUNTS"], common["_SW_NGS_VALUES"], common["_SW_NGM_VALUES"],
         common["_SW_NGN_VALUES"], 14, 16, _SW_RECORDS, "RRTMG_SW_DATA"),
    ):
        rwgt = _rwgt(counts, ngm, ngn, common["_RRTMG_WT_VALUES"])
        t[f"{side}.rwgt"] = rwgt
        t[f"{side}.ngc"] = i32(counts)
        t[f"{side}.ngs"] = i32(ngs)
        t[f"{side}.ngn"] = i32(ngn)
        raw = _read_records(data / "rrtmg" / fname, records)
        for ib in range(nb):
            t.update(_compress(raw[first + ib], ib, counts, ngs, ngn, rwgt, f"{side}{first + ib}"))

    with np.load(data / "rrtmg_lw_setcoef_tables.npz") as d:
        for k in ("pref", "preflog", "tref", "chi_mls", "totplnk", "totplk16"):
            t[f"lw.{k}"] = f32(d[k])
    with np.load(data / "rrtmg_lw_cloud_tables.npz") as d:
        for k in d.files:
            t[f"lw.{k}"] = f32(d[k]).reshape(-1) if np.ndim(d[k]) == 0 else f32(d[k])
    with np.load(data / "rrtmg_lw_pade_tables.npz") as d:
        for k in ("bpade", "tau_tbl", "exp_tbl", "tfn_tbl"):
            t[f"lw.pade_{k}"] = f32(d[k]).reshape(-1)
    with np.load(data / "rrtmg_sw_cloud_tables.npz") as d:
        for k in d.files:
            t[f"sw.{k}"] = f32(d[k])
    with np.load(data / "rrtmg_sw_pade_tables.npz") as d:
        for k in ("bpade", "tau_tbl", "exp_tbl"):
            t[f"sw.pade_{k}"] = f32(d[k]).reshape(-1)
    return t


def write_blob(tables: dict, path: str | Path) -> None:
    names = sorted(tables)
    header = bytearray(MAGIC + struct.pack("<II", VERSION, len(names)))
    entry_size = 48 + 4 + 4 + 16 + 8 + 8
    data_start = len(header) + entry_size * len(names)
    data_start = (data_start + 255) // 256 * 256
    body = bytearray()
    entries = bytearray()
    for name in names:
        arr = np.ascontiguousarray(tables[name])
        if arr.dtype == np.float32:
            code = 0
        elif arr.dtype == np.int32:
            code = 1
        elif arr.dtype == np.float64:
            code = 2
        elif arr.dtype == np.uint64:
            code = 3
        else:
            raise TypeError(f"{name}: unsupported dtype {arr.dtype}")
        if arr.ndim > 4 or len(name) >= 48:
            raise ValueError(name)
        shape = list(arr.shape) + [1] * (4 - arr.ndim)
        pad = (-len(body)) % 256
        body += b"\0" * pad
        offset = data_start + len(body)
        raw = arr.astype(arr.dtype.newbyteorder("<")).tobytes()
        body += raw
        entries += name.encode().ljust(48, b"\0")
        entries += struct.pack("<II4IQQ", code, arr.ndim, *shape, offset, len(raw))
    out = header + entries
    out += b"\0" * (data_start - len(out))
    out += body
    Path(path).write_bytes(bytes(out))


def read_blob(path: str | Path) -> dict:
    raw = Path(path).read_bytes()
    if raw[:8] != MAGIC:
        raise ValueError(f"{path}: not an RRTMG table blob")
    version, count = struct.unpack_from("<II", raw, 8)
    if version != VERSION:
        raise ValueError(f"{path}: blob version {version}, expected {VERSION}")
    pos = 16
    out = {}
    for _ in range(count):
        name = raw[pos:pos + 48].split(b"\0", 1)[0].decode()
        code, ndim, s0, s1, s2, s3, offset, nbytes = struct.unpack_from("<II4IQQ", raw, pos + 48)
        pos += 88
        dt = {0: np.float32, 1: np.int32, 2: np.float64, 3: np.uint64}[code]
        out[name] = np.frombuffer(raw, dtype=dt, count=nbytes // np.dtype(dt).itemsize,
                                  offset=offset).reshape((s0, s1, s2, s3)[:ndim])
    return out


DEFAULT_BLOB = Path(__file__).resolve().parent / "data" / "rrtmg_tables.bin"
# entries added after the first blob layout: a blob without them is rebuilt
REQUIRED_ENTRIES = frozenset({"svml.sinf", "svml.cosf", "lw.ngn", "sw.ngn"})


def _blob_names(path: Path) -> set:
    try:
        raw = Path(path).read_bytes()
        _, count = struct.unpack_from("<II", raw, 8)
        return {raw[16 + 88 * i:16 + 88 * i + 48].split(b"\0", 1)[0].decode() for i in range(count)}
    except (OSError, struct.error, UnicodeDecodeError):
        return set()


def ensure_blob(physics_dir: str | Path | None = None, path: str | Path = DEFAULT_BLOB) -> Path:
    """Build the blob from a WRF-JAX physics directory if it is missing or lacks an entry
    of REQUIRED_ENTRIES."""
    path = Path(path)
    if path.exists() and (physics_dir is None or REQUIRED_ENTRIES <= _blob_names(path)):
        return path
    if physics_dir is None:
        raise FileNotFoundError(
            f"{path} is missing; build it with tables.ensure_blob(<wrf_jax/physics dir>)")
    path.parent.mkdir(parents=True, exist_ok=True)
    write_blob(build_tables(physics_dir), path)
    return path
