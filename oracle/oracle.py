"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle (``liboracle_rrtmg.so``, sources beside this file) restates WRF-JAX's
RRTMG LW/SW radiation path in plain C with the reference's binary32 rounding.
Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use
it, as the checker; the product path never imports this module.

``lwrad(**kw)`` / ``swrad(**kw)`` take the reference's keyword arguments
(``rrtmg_lwrad_wrf_columns``, module_ra_rrtmg_lw.py:6789;
``rrtmg_swrad_wrf_columns``, module_ra_rrtmg_sw.py:2386) in the WRF runtime
layout and return dicts keyed by the reference's result field names.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle_rrtmg.so"

_OUT_FIELDS = ("rthraten", "rthratenc", "up_top", "upc_top", "dn_top", "dnc_top", "up_sfc",
               "upc_sfc", "dn_sfc", "dnc_sfc", "swddir", "swddni", "swddif", "swddirc",
               "swddnic", "taug", "fracs_or_taur", "cldfmc", "taucmc", "uflx", "dflx", "uflxc",
               "dflxc", "hr", "hrc")


def _structs(real):
    """ora_in / ora_out with `real` (c_float, or c_double in the binary64 build) as
    the element type of the arrays and of the gas scalars."""
    ptr = ctypes.POINTER(real)

    class In(ctypes.Structure):
        _fields_ = [("ncol", ctypes.c_int), ("nk", ctypes.c_int)] + [
            (n, ptr) for n in ("p3d", "pi3d", "t3d", "qv", "qc", "qi", "qs", "cldfra", "o3",
                               "re_cloud", "re_ice", "re_snow", "p8w", "t8w", "tsk", "emiss",
                               "albedo", "coszr", "xland", "xice", "snow")
        ] + [("p_top", ctypes.c_double)] + [
            (n, real) for n in ("co2", "n2o", "ch4", "cfc11", "cfc12", "solcon")
        ] + [(n, ctypes.c_int) for n in ("has_reqc", "has_reqi", "has_reqs", "icloud", "cldovrlp",
                                         "fp64_steps")] + [
            (n, ptr) for n in ("alswvisdir", "alswvisdif", "alswnirdir", "alswnirdif")]

    class Out(ctypes.Structure):
        _fields_ = [(n, ptr) for n in _OUT_FIELDS]

    return In, Out


_In, _Out = _structs(ctypes.c_float)
_In64, _Out64 = _structs(ctypes.c_double)

COUNT_LIB_PATH = HERE / "liboracle_rrtmg_count.so"
F64_LIB_PATH = HERE / "liboracle_rrtmg_f64.so"


def build(force: bool = False, counted: bool = False, binary64: bool = False) -> Path:
    """Compile the oracle with its Makefile (gcc, no GPU needed); ``counted``
    builds the FLOP-counting variant (flop_count.h), ``binary64`` the variant
    that does every operation in binary64 (fp64.h) instead."""
    srcs = [HERE / n for n in ("oracle_common.c", "oracle_lw.c", "oracle_sw.c", "oracle.h",
                                "oracle_internal.h")]
    lib = COUNT_LIB_PATH if counted else (F64_LIB_PATH if binary64 else LIB_PATH)
    if counted:
        srcs += [HERE / "flop_count.h", HERE / "flop_count.cc"]
    if binary64:
        srcs += [HERE / "fp64.h"]
    if force or not lib.exists() or any(s.stat().st_mtime > lib.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE), lib.name], check=True)
    return lib


class Oracle:
    """Loaded oracle library plus one table blob."""

    def __init__(self, blob_path: str | os.PathLike, nthreads: int | None = None, counted: bool = False,
                 binary64: bool = False):
        """``binary64``: the build whose arithmetic is binary64 throughout (an
        FP64 run of the path); its inputs are widened from binary32 and its
        outputs are float64 arrays."""
        self.lib = ctypes.CDLL(str(build(counted=counted, binary64=binary64)))
        self.counted = counted
        self.binary64 = binary64
        self._dtype = np.float64 if binary64 else np.float32
        self._In, self._Out = (_In64, _Out64) if binary64 else (_In, _Out)
        self._ptr = ctypes.POINTER(ctypes.c_double if binary64 else ctypes.c_float)
        if counted:
            nthreads = 1  # the counters are per thread
            self.lib.ora_flop_counts_take.restype = None
            self.lib.ora_flop_counts_take.argtypes = [ctypes.POINTER(ctypes.c_ulonglong)]
        self.lib.ora_tables_load.restype = ctypes.c_void_p
        self.lib.ora_tables_load.argtypes = [ctypes.c_char_p]
        self.lib.ora_tables_free.argtypes = [ctypes.c_void_p]
        for name in ("ora_lw_columns", "ora_sw_columns"):
            fn = getattr(self.lib, name)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_void_p, ctypes.POINTER(self._In), ctypes.POINTER(self._Out), ctypes.c_int]
        self.lib.ora_lw_nlayers.restype = ctypes.c_int
        self.lib.ora_lw_nlayers.argtypes = [ctypes.c_double, ctypes.c_int]
        self.tables = self.lib.ora_tables_load(str(blob_path).encode())
        if not self.tables:
            raise RuntimeError(f"oracle could not load table blob {blob_path}")
        self.nthreads = nthreads or os.cpu_count() or 1

    def __del__(self):
        tables = getattr(self, "tables", None)
        if tables:
            self.lib.ora_tables_free(tables)
            self.tables = None

    def take_counts(self) -> dict:
        """Operations counted since the last call (counted build only): binary32
        add (incl. subtract), mul, div, sqrt, exp, log, pow."""
        buf = (ctypes.c_ulonglong * 7)()
        self.lib.ora_flop_counts_take(buf)
        return dict(zip(("add", "mul", "div", "sqrt", "exp", "log", "pow"), (int(v) for v in buf)))

    # ------------------------------------------------------------------
    def _columns(self, a):  # (nx, nz, ny) -> (ncol, nz), column index = i*ny + j
        a = np.asarray(np.asarray(a, np.float32), self._dtype)
        return np.ascontiguousarray(np.swapaxes(a, 1, 2).reshape(-1, a.shape[1]))

    def _flat2d(self, a):
        return np.ascontiguousarray(np.asarray(np.asarray(a, np.float32), self._dtype).reshape(-1))

    def _inputs(self, kw):
        t3d = np.asarray(kw["t3d"])
        nx, nk, ny = t3d.shape
        ncol = nx * ny
        keep = {}

        def ptr(a):
            keep[id(a)] = a
            return a.ctypes.data_as(self._ptr)

        s = self._In()
        s.ncol, s.nk = ncol, nk
        for name, key in (("p3d", "p3d"), ("pi3d", "pi3d"), ("t3d", "t3d"), ("qv", "qv3d"),
                          ("qc", "qc3d"), ("qi", "qi3d"), ("qs", "qs3d"), ("cldfra", "cldfra3d"),
                          ("o3", "o33d"), ("re_cloud", "re_cloud"), ("re_ice", "re_ice"),
                          ("re_snow", "re_snow"), ("p8w", "p8w"), ("t8w", "t8w")):
            setattr(s, name, ptr(self._columns(kw[key])))
        zeros2 = np.zeros(ncol, self._dtype)
        for name in ("tsk", "emiss", "albedo", "coszr", "xland", "xice", "snow"):
            setattr(s, name, ptr(self._flat2d(kw[name]) if name in kw else zeros2))
        s.p_top = float(kw.get("p_top", 5000.0))
        s.co2 = np.float32(kw["co2vmr"])
        s.n2o = np.float32(kw["n2ovmr"])
        s.ch4 = np.float32(kw["ch4vmr"])
        s.cfc11 = np.float32(kw.get("cfc11vmr", 0.0))
        s.cfc12 = np.float32(kw.get("cfc12vmr", 0.0))
        s.solcon = np.float32(kw.get("solcon", 0.0))
        s.fp64_steps = int(kw.get("fp64_steps", 0))
        # Noah-MP albedos (sf_surface_physics == 8, all four given; sw:2521)
        albs = ("alswvisdir", "alswvisdif", "alswnirdir", "alswnirdif")
        if int(kw.get("sf_surface_physics", 2)) == 8 and all(kw.get(n) is not None for n in albs):
            for n in albs:
                setattr(s, n, ptr(self._flat2d(kw[n])))
        s.has_reqc = int(kw.get("has_reqc", 1))
        s.has_reqi = int(kw.get("has_reqi", 1))
        s.has_reqs = int(kw.get("has_reqs", 1))
        s.icloud = int(kw.get("icloud", 1))
        s.cldovrlp = int(kw.get("cldovrlp", 2))
        return s, keep, (nx, nk, ny)

    def _outputs(self, ncol, nk, nlay, ngpt, diagnostics):
        bufs = {}
        o = self._Out()
        sizes = dict(rthraten=ncol * nk, rthratenc=ncol * nk)
        for n in ("up_top", "upc_top", "dn_top", "dnc_top", "up_sfc", "upc_sfc", "dn_sfc",
                  "dnc_sfc", "swddir", "swddni", "swddif", "swddirc", "swddnic"):
            sizes[n] = ncol
        if diagnostics:
            sizes.update(taug=ncol * nlay * ngpt, fracs_or_taur=ncol * nlay * ngpt,
                         cldfmc=ncol * ngpt * nlay, taucmc=ncol * ngpt * nlay,
                         uflx=ncol * (nlay + 1), dflx=ncol * (nlay + 1), uflxc=ncol * (nlay + 1),
                         dflxc=ncol * (nlay + 1), hr=ncol * nlay, hrc=ncol * nlay)
        for n, size in sizes.items():
            bufs[n] = np.zeros(size, self._dtype)
            setattr(o, n, bufs[n].ctypes.data_as(self._ptr))
        return o, bufs

    @staticmethod
    def _unflat3(a, nx, ny):
        return np.swapaxes(a.reshape(nx, ny, -1), 1, 2)

    # ------------------------------------------------------------------
    def lwrad(self, diagnostics: bool = False, **kw) -> dict:
        s, keep, (nx, nk, ny) = self._inputs(kw)
        ncol = nx * ny
        nlay = self.lib.ora_lw_nlayers(float(kw.get("p_top", 5000.0)), nk)
        o, b = self._outputs(ncol, nk, nlay, 140, diagnostics)
        rc = self.lib.ora_lw_columns(self.tables, ctypes.byref(s), ctypes.byref(o), self.nthreads)
        if rc != 0:
            raise RuntimeError(f"oracle LW failed with status {rc}")
        two = lambda a: a.reshape(nx, ny)
        zeros = np.zeros((nx, ny), self._dtype)
        out = dict(
            rthratenlw=self._unflat3(b["rthraten"], nx, ny),
            rthratenlwc=self._unflat3(b["rthratenc"], nx, ny),
            lwupt=two(b["up_top"]), lwuptc=two(b["upc_top"]), lwuptcln=zeros,
            lwdnt=two(b["dn_top"]), lwdntc=two(b["dnc_top"]), lwdntcln=zeros,
            lwupb=two(b["up_sfc"]), lwupbc=two(b["upc_sfc"]), lwupbcln=zeros,
            lwdnb=two(b["dn_sfc"]), lwdnbc=two(b["dnc_sfc"]), lwdnbcln=zeros,
            glw=two(b["dn_sfc"]), olr=two(b["up_top"]),
            lwcf=two(b["upc_top"] - b["up_top"]),
        )
        if diagnostics:
            out["diag"] = dict(
                taug=b["taug"].reshape(ncol, nlay, 140), fracs=b["fracs_or_taur"].reshape(ncol, nlay, 140),
                cldfmc=b["cldfmc"].reshape(ncol, 140, nlay), taucmc=b["taucmc"].reshape(ncol, 140, nlay),
                uflx=b["uflx"].reshape(ncol, nlay + 1), dflx=b["dflx"].reshape(ncol, nlay + 1),
                uflxc=b["uflxc"].reshape(ncol, nlay + 1), dflxc=b["dflxc"].reshape(ncol, nlay + 1),
                hr=b["hr"].reshape(ncol, nlay), hrc=b["hrc"].reshape(ncol, nlay))
        return out

    def swrad(self, diagnostics: bool = False, **kw) -> dict:
        s, keep, (nx, nk, ny) = self._inputs(kw)
        ncol = nx * ny
        nlay = nk + 1
        o, b = self._outputs(ncol, nk, nlay, 112, diagnostics)
        rc = self.lib.ora_sw_columns(self.tables, ctypes.byref(s), ctypes.byref(o), self.nthreads)
        if rc != 0:
            raise RuntimeError(f"oracle SW failed with status {rc}")
        two = lambda a: a.reshape(nx, ny)
        zeros = np.zeros((nx, ny), self._dtype)
        coszr = self._flat2d(kw["coszr"])
        day = coszr > 0.0
        up_t, upc_t, dn_t, dnc_t = b["up_top"], b["upc_top"], b["dn_top"], b["dnc_top"]
        swcf = np.where(day, (dn_t - up_t) - (dnc_t - upc_t), 0.0).astype(self._dtype)
        gsw = np.where(day, b["dn_sfc"] - b["up_sfc"], 0.0).astype(self._dtype)
        out = dict(
            rthratensw=self._unflat3(b["rthraten"], nx, ny),
            rthratenswc=self._unflat3(b["rthratenc"], nx, ny),
            swupt=two(up_t), swuptc=two(upc_t), swuptcln=zeros,
            swdnt=two(dn_t), swdntc=two(dnc_t), swdntcln=zeros,
            swupb=two(b["up_sfc"]), swupbc=two(b["upc_sfc"]), swupbcln=zeros,
            swdnb=two(b["dn_sfc"]), swdnbc=two(b["dnc_sfc"]), swdnbcln=zeros,
            swcf=two(swcf), gsw=two(gsw),
            swddir=two(b["swddir"]), swddni=two(b["swddni"]), swddif=two(b["swddif"]),
            swdownc=two(b["dnc_sfc"]), swddnic=two(b["swddnic"]), swddirc=two(b["swddirc"]),
            coszr=two(coszr),
        )
        if diagnostics:
            out["diag"] = dict(
                taug=b["taug"].reshape(ncol, nlay, 112), taur=b["fracs_or_taur"].reshape(ncol, nlay, 112),
                cldfmc=b["cldfmc"].reshape(ncol, 112, nlay), taucmc=b["taucmc"].reshape(ncol, 112, nlay),
                uflx=b["uflx"].reshape(ncol, nlay + 1), dflx=b["dflx"].reshape(ncol, nlay + 1),
                uflxc=b["uflxc"].reshape(ncol, nlay + 1), dflxc=b["dflxc"].reshape(ncol, nlay + 1),
                hr=b["hr"].reshape(ncol, nlay), hrc=b["hrc"].reshape(ncol, nlay))
        return out
