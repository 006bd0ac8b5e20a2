"""Radiation over several GPUs: one process per GPU, south-north rows split across ranks.

The reference spreads a radiation call over its configured GPUs in whole
batches of south-north rows (``batch_partitions``, src/wrf_jax/core/devices.py:29-41;
``_run_radiation_columns_chunked``, src/wrf_jax/runtime.py:5361-5402) and
concatenates the results in row order.  Here each rank of a
``torch.distributed`` job takes its rows of the same partition and calls the
kernels on them; columns are independent and the McICA stream is seeded per
column from its own pressures, so the results do not depend on the split.
The one collective is the gather of the outputs, for callers that want whole
fields on every rank; ``max_over_ranks`` is the timing reduction.
"""

from __future__ import annotations

from typing import Any, Callable, Mapping


def batch_partitions(length: int, batch_size: int, device_count: int) -> tuple:
    """Whole batches of ``batch_size`` rows spread over at most ``device_count``
    ranks, as contiguous (start, stop) ranges (core/devices.py:29-41)."""
    if min(length, batch_size, device_count) < 1:
        raise ValueError("positive length, batch size and device count required")
    batches = -(-length // batch_size)
    used = min(device_count, batches)
    per, extra = divmod(batches, used)
    ranges, start = [], 0
    for r in range(used):
        stop = start + (per + (1 if r < extra else 0)) * batch_size
        ranges.append((start, min(stop, length)))
        start = stop
    return tuple(ranges)


def rank_rows(ny: int, world: int, rank: int, rows_per_batch: int = 1) -> tuple[int, int]:
    """South-north rows [j0, j1) of ``rank``; ranks beyond the batches get an empty range."""
    ranges = batch_partitions(ny, rows_per_batch, world)
    return ranges[rank] if rank < len(ranges) else (ny, ny)


def slice_rows(value: Any, nx: int, ny: int, j0: int, j1: int) -> Any:
    """Rows j0..j1 of a WRF-layout array ((nx, nz, ny) or (nx, ny)); other values
    pass through (runtime.py:5123-5131)."""
    shape = getattr(value, "shape", None)
    if shape is None:
        return value
    if len(shape) == 3 and shape[0] == nx and shape[2] == ny:
        return value[:, :, j0:j1]
    if len(shape) == 2 and shape[0] == nx and shape[1] == ny:
        return value[:, j0:j1]
    return value


def _as_tensor(v):
    import numpy as np
    import torch

    if isinstance(v, torch.Tensor):
        return v
    return torch.from_numpy(np.ascontiguousarray(v))


def gather_rows(local: Mapping[str, Any], ranges: tuple, ny: int, group=None) -> dict:
    """Every rank's row slabs of each field, concatenated in row order on every
    rank (an all-gather of slabs padded to the widest one, then trimmed)."""
    import torch
    import torch.distributed as dist

    out = {}
    world = dist.get_world_size(group)
    widths = [b - a for a, b in ranges] + [0] * (world - len(ranges))
    wmax = max(widths)
    for name, value in local.items():
        t = _as_tensor(value).contiguous()
        pad = list(t.shape)
        pad[-1] = wmax
        buf = torch.zeros(pad, dtype=t.dtype, device=t.device)
        buf[..., : t.shape[-1]] = t
        parts = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(parts, buf, group=group)
        out[name] = torch.cat([p[..., :w] for p, w in zip(parts, widths) if w > 0], dim=-1)
        if out[name].shape[-1] != ny:
            raise RuntimeError(f"{name}: gathered {out[name].shape[-1]} rows, expected {ny}")
    return out


def max_over_ranks(value: float, group=None, device=None) -> float:
    """The largest of every rank's value (the multi-GPU step time is the slowest rank's)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def sharded_call(call: Callable[..., Any], kwargs: Mapping[str, Any], *, rank: int, world: int,
                 rows_per_batch: int = 1, gather: bool = True, group=None, device: int | None = None):
    """Run ``call`` (e.g. ``rrtmg.rrtmg_lwrad_wrf_columns``) on this rank's rows of
    the domain in ``kwargs``.  Returns (rows, result): result holds this rank's
    slab of every output field, or with ``gather`` the whole fields on every rank.
    A gather needs rows on every rank; the check is the same on all ranks, so
    they all raise before any collective.

    Device: the radiation calls run on the context they are given, else on
    the process's current CUDA device (``rrtmg.default_context``).  With one
    process per GPU, pass ``device`` (normally the local rank) or call
    ``torch.cuda.set_device(local_rank)`` first; otherwise every rank uses
    GPU 0.  With ``device`` the call runs under ``torch.cuda.device(device)``
    and the caller's current device is restored afterwards."""
    if device is not None:
        import torch

        with torch.cuda.device(int(device)):
            return sharded_call(call, kwargs, rank=rank, world=world, rows_per_batch=rows_per_batch,
                                gather=gather, group=group)
    t3d = kwargs["t3d"]
    nx, ny = int(t3d.shape[0]), int(t3d.shape[2])
    ranges = batch_partitions(ny, rows_per_batch, world)
    if gather and len(ranges) < world:
        raise ValueError(f"{world} ranks but {len(ranges)} row batches: lower world or rows_per_batch")
    j0, j1 = ranges[rank] if rank < len(ranges) else (ny, ny)
    local = None
    if j1 > j0:
        res = call(**{k: slice_rows(v, nx, ny, j0, j1) for k, v in kwargs.items()})
        local = res._asdict() if hasattr(res, "_asdict") else dict(res)
    if not gather:
        return (j0, j1), local
    return (j0, j1), gather_rows(local, ranges, ny, group)
