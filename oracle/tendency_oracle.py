"""CPU oracle of the radiation tendency chain (test infrastructure only).

A numpy restatement of what follows the RRTMG calls for the potential
temperature:

* ``rthraten = rthratenlw + rthratensw``  (src/wrf_jax/runtime.py:7946);
* mass coupling ``rthraten * (c1[k] * mut + c2[k])`` over the tile
  (``calculate_phy_tend`` / ``multiply_3d``, src/wrf_jax/dyn_em/module_em.py:577-602,
  621-622), each product and sum rounded to binary32;
* accumulation into ``rt_tendf`` over the tile less the specified / nested
  boundary rows (``phy_ra_ten`` -> ``add_a2a`` / ``_a2a_bounds``,
  src/wrf_jax/physics/module_physics_addtendc.py:131-204, 542-590).

Arrays are memory-sized: (ime-ims+1, kme-kms+1, jme-jms+1), c1/c2 (kme-kms+1),
mut (ime-ims+1, jme-jms+1).  Only tests use this module, as the checker.
"""

from __future__ import annotations

import numpy as np

BOUND_NAMES = ("ids", "ide", "jds", "jde", "kds", "kde", "ims", "ime", "jms", "jme", "kms", "kme",
               "its", "ite", "jts", "jte", "kts", "kte")


def tile_region(b: dict) -> tuple[slice, slice, slice]:
    """calculate_phy_tend's multiply region (module_em.py:577-593)."""
    itf = min(b["ite"], b["ide"] - 1)
    jtf = min(b["jte"], b["jde"] - 1)
    ktf = min(b["kte"], b["kde"] - 1)
    if b["its"] > itf or b["jts"] > jtf or b["kts"] > ktf:
        return slice(0, 0), slice(0, 0), slice(0, 0)
    return (slice(b["its"] - b["ims"], itf - b["ims"] + 1), slice(b["kts"] - b["kms"], ktf - b["kms"] + 1),
            slice(b["jts"] - b["jms"], jtf - b["jms"] + 1))


def a2a_region(b: dict) -> tuple[slice, slice, slice]:
    """add_a2a's region (module_physics_addtendc.py:131-170)."""
    i0, i1 = b["its"], min(b["ite"], b["ide"] - 1)
    j0, j1 = b["jts"], min(b["jte"], b["jde"] - 1)
    ktf = min(b["kte"], b["kde"] - 1)
    if b.get("specified") or b.get("nested"):
        i0, i1 = max(b["ids"] + 1, b["its"]), min(b["ide"] - 2, b["ite"])
        j0, j1 = max(b["jds"] + 1, b["jts"]), min(b["jde"] - 2, b["jte"])
    if b.get("periodic_x"):
        i0, i1 = b["its"], min(b["ite"], b["ide"] - 1)
    return (slice(i0 - b["ims"], max(i1 - b["ims"] + 1, 0)), slice(b["kts"] - b["kms"], ktf - b["kms"] + 1),
            slice(j0 - b["jms"], max(j1 - b["jms"] + 1, 0)))


def radiation_tendency(lw, sw, c1, c2, mut, rt_tendf, b: dict, couple: bool = True):
    """(rthraten after coupling, rt_tendf after accumulation), binary32."""
    f = np.float32
    r = (np.asarray(lw, f) + np.asarray(sw, f)).astype(f)
    if couple:
        i, k, j = tile_region(b)
        factor = (np.asarray(c1, f)[k][None, :, None] * np.asarray(mut, f)[i, j][:, None, :]).astype(f)
        factor = (factor + np.asarray(c2, f)[k][None, :, None]).astype(f)
        r[i, k, j] = (r[i, k, j] * factor).astype(f)
    t = np.array(rt_tendf, dtype=f, copy=True)
    region = a2a_region(b)
    t[region] = (t[region] + r[region]).astype(f)
    return r, t
