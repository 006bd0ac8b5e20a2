"""rrtmg_b200: WRF-JAX's RRTMG longwave + shortwave radiation path on NVIDIA B200.

The package exposes the reference's two radiation calls with the same keyword
signature and result fields:

* ``rrtmg_lwrad_wrf_columns(**kw) -> RrtmgLwWrfColumnResult``
* ``rrtmg_swrad_wrf_columns(**kw) -> RrtmgSwWrfColumnResult``

Both run as hand-written sm_100a CUDA kernels behind the C-ABI declared in
``include/rrtmg_b200.h`` (``librrtmg_b200.so``).  There is no CPU fallback: if
the shared library or a CUDA device is missing the calls raise.
"""

from importlib import import_module

_EXPORTS = {
    "RrtmgLwWrfColumnResult": "rrtmg",
    "RrtmgSwWrfColumnResult": "rrtmg",
    "RrtmgContext": "rrtmg",
    "rrtmg_lwrad_wrf_columns": "rrtmg",
    "rrtmg_swrad_wrf_columns": "rrtmg",
}
__all__ = sorted(_EXPORTS)


def __getattr__(name):
    if name not in _EXPORTS:
        raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
    value = getattr(import_module(f".{_EXPORTS[name]}", __name__), name)
    globals()[name] = value
    return value
