"""Radiation heating applied to the potential-temperature tendency, on B200.

After its RRTMG calls WRF-JAX forms ``rthraten = rthratenlw + rthratensw``
(src/wrf_jax/runtime.py:7946), couples it with the column mass in
``calculate_phy_tend`` (src/wrf_jax/dyn_em/module_em.py:462, 621-622) and adds
it to ``t_tendf`` in ``phy_ra_ten`` (src/wrf_jax/physics/module_physics_addtendc.py:542).
``radiation_tendency`` does the three in one pass over the arrays
(``rrtmg_radiation_tendency``, include/rrtmg_tendency.h); ``phy_ra_ten``
mirrors the reference's function of that name.  Results are bit-identical.

Arrays are float32 in WRF memory order, (ime-ims+1, kme-kms+1, jme-jms+1);
numpy arrays are copied to the GPU and results copied back, torch CUDA tensors
stay on the GPU.  There is no CPU path.
"""

from __future__ import annotations

import ctypes

from . import _capi
from .rrtmg import RrtmgError, _as_device

_BOUNDS = ("ids", "ide", "jds", "jde", "kds", "kde", "ims", "ime", "jms", "jme", "kms", "kme",
           "its", "ite", "jts", "jte", "kts", "kte")


def _flag(config_flags, name: str) -> int:
    if hasattr(config_flags, "get"):
        return int(bool(config_flags.get(name, False)))
    return int(bool(getattr(config_flags, name, False)))


def bounds(config_flags, **b) -> "_capi.TendencyBounds":
    """rrtmg_tendency_bounds from WRF index keywords; ``ime``/``jme``/``kme``
    default to the tile's memory extents as the reference's keywords do not
    always carry them."""
    vals = {k: int(b[k]) for k in _BOUNDS if b.get(k) is not None}
    missing = [k for k in _BOUNDS if k not in vals]
    if missing:
        raise ValueError(f"missing bounds: {missing}")
    return _capi.TendencyBounds(**vals, specified=_flag(config_flags, "specified"),
                                nested=_flag(config_flags, "nested"), periodic_x=_flag(config_flags, "periodic_x"))


def _shape(tb) -> tuple:
    return (tb.ime - tb.ims + 1, tb.kme - tb.kms + 1, tb.jme - tb.jms + 1)


def _check(st: int, what: str) -> None:
    if st != 0:
        raise RrtmgError(st, f"{what} rejected its arguments (bounds, shapes or pointers)")


def radiation_tendency(rthratenlw, rthratensw, c1, c2, mut, rt_tendf, config_flags, *, couple: bool = True,
                       stream=None, **bounds_kw):
    """(rthraten coupled, rt_tendf updated): the LW + SW sum, the mass coupling
    over the tile and its accumulation into ``rt_tendf`` over the a2a region.
    ``rt_tendf`` is not modified; a new array is returned, as the reference's
    functions do."""
    import torch

    tb = bounds(config_flags, **bounds_kw)
    shape = _shape(tb)
    dev = torch.cuda.current_device()
    d, host = _as_device(dict(lw=rthratenlw, sw=rthratensw, c1=c1, c2=c2, mut=mut, t=rt_tendf), dev)
    for k in ("lw", "sw", "t"):
        if tuple(d[k].shape) != shape:
            raise ValueError(f"3-D arrays must have the memory shape {shape}, got {tuple(d[k].shape)}")
    if couple and (d["c1"].numel() != shape[1] or d["c2"].numel() != shape[1]
                   or tuple(d["mut"].shape) != (shape[0], shape[2])):
        raise ValueError("c1/c2 must have kme-kms+1 values and mut (ime-ims+1, jme-jms+1)")
    r = torch.empty(shape, dtype=torch.float32, device=d["lw"].device)
    t = d["t"].clone()
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    lib = _capi.load()
    _check(lib.rrtmg_radiation_tendency(ctypes.byref(tb), d["lw"].data_ptr(), d["sw"].data_ptr(),
                                        d["c1"].data_ptr(), d["c2"].data_ptr(), d["mut"].data_ptr(), int(couple),
                                        r.data_ptr(), t.data_ptr(), ctypes.c_void_p(s)), "rrtmg_radiation_tendency")
    if host:
        torch.cuda.current_stream().synchronize()
        return r.cpu().numpy(), t.cpu().numpy()
    return r, t


def phy_ra_ten(config_flags, rt_tendf, rthraten, *, stream=None, **bounds_kw):
    """WRF phy_ra_ten (module_physics_addtendc.py:542): rt_tendf + rthraten over
    the a2a region, as a new array."""
    import torch

    tb = bounds(config_flags, **bounds_kw)
    shape = _shape(tb)
    dev = torch.cuda.current_device()
    d, host = _as_device(dict(t=rt_tendf, r=rthraten), dev)
    for k in ("t", "r"):
        if tuple(d[k].shape) != shape:
            raise ValueError(f"arrays must have the memory shape {shape}, got {tuple(d[k].shape)}")
    t = d["t"].clone()
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    _check(_capi.load().rrtmg_phy_ra_ten(ctypes.byref(tb), t.data_ptr(), d["r"].data_ptr(), ctypes.c_void_p(s)),
           "rrtmg_phy_ra_ten")
    if host:
        torch.cuda.current_stream().synchronize()
        return t.cpu().numpy()
    return t
