"""Multi-rank radiation on the CPU: two gloo ranks split a domain's south-north
rows as the reference's batch_partitions does, each runs its slab through the
CPU oracle (standing in for the GPU kernels, which need a device), and the
gathered fields equal the whole-domain result bit for bit (columns are
independent; McICA is seeded per column).  Also the timing reduction and the
partition arithmetic against the reference's own function."""

from __future__ import annotations

import ast
import os
import socket
import sys

import numpy as np
import pytest

from conftest import REPO, REFERENCE_PHYSICS


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, blob: str, out_dir: str, rows_per_batch: int) -> None:
    import torch.distributed as dist

    sys.path.insert(0, str(REPO / "tests"))
    sys.path.insert(0, str(REPO / "oracle"))
    import conftest
    conftest.load_package()
    import oracle
    from wrf_jax_b200 import sharding, synthetic

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ora = oracle.Oracle(blob, nthreads=1)
        st = synthetic.make_columns(3, 7, 44, seed=21)
        for side, kw in (("lw", st.lw_kwargs()), ("sw", st.sw_kwargs())):
            call = ora.lwrad if side == "lw" else ora.swrad
            (j0, j1), full = sharding.sharded_call(call, kw, rank=rank, world=world, rows_per_batch=rows_per_batch)
            np.savez(os.path.join(out_dir, f"{side}_{rank}.npz"), j=np.asarray([j0, j1]),
                     **{k: v.numpy() for k, v in full.items()})
        slowest = sharding.max_over_ranks(10.0 + rank)
        np.save(os.path.join(out_dir, f"max_{rank}.npy"), np.asarray(slowest))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("rows_per_batch", [1, 2])
def test_two_rank_split_equals_whole_domain(pkg, blob_path, oracle, tmp_path, rows_per_batch):
    import torch.multiprocessing as mp
    from wrf_jax_b200 import synthetic

    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(blob_path), str(tmp_path), rows_per_batch), nprocs=2,
                       join=True, start_method="spawn")
    st = synthetic.make_columns(3, 7, 44, seed=21)
    want = {"lw": oracle.lwrad(**st.lw_kwargs()), "sw": oracle.swrad(**st.sw_kwargs())}
    spans = []
    for rank in range(2):
        for side in ("lw", "sw"):
            with np.load(tmp_path / f"{side}_{rank}.npz") as got:
                spans.append(tuple(got["j"]))
                for name, value in want[side].items():
                    np.testing.assert_array_equal(got[name], value, err_msg=f"rank {rank} {side} {name}")
        assert float(np.load(tmp_path / f"max_{rank}.npy")) == 11.0
    # both ranks had rows, and together they cover the domain
    assert spans[0][0] == 0 and spans[2][1] == 7 and spans[0][1] == spans[2][0]


def test_partitions_match_the_reference(pkg):
    from wrf_jax_b200 import sharding
    path = REFERENCE_PHYSICS.parent / "core" / "devices.py"
    if not path.exists():
        pytest.skip("WRF-JAX sources are not on this machine")
    tree = ast.parse(path.read_text())
    node = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "batch_partitions")
    ns: dict = {}
    exec(compile(ast.Module(body=[node], type_ignores=[]), str(path), "exec"), ns)
    for length in (1, 5, 7, 64, 425, 1000):
        for batch in (1, 2, 3, 16, 1000):
            for devices in (1, 2, 3, 4, 8):
                assert sharding.batch_partitions(length, batch, devices) == ns["batch_partitions"](length, batch, devices)


def test_gather_rejects_more_ranks_than_batches(pkg):
    from wrf_jax_b200 import sharding
    kw = {"t3d": np.zeros((2, 4, 3), np.float32)}
    with pytest.raises(ValueError):
        sharding.sharded_call(lambda **k: {}, kw, rank=0, world=4, rows_per_batch=1)
    assert sharding.rank_rows(3, 4, 3) == (3, 3)
    assert sharding.slice_rows(np.zeros((2, 5, 3)), 2, 3, 1, 2).shape == (2, 5, 1)
    assert sharding.slice_rows(np.zeros((2, 3)), 2, 3, 0, 2).shape == (2, 2)


@pytest.mark.gpu
def test_rank_slabs_on_one_gpu_equal_whole_domain(pkg):
    """The CUDA kernels through sharded_call: both ranks' row ranges of a
    two-rank split (run one after the other on one GPU, gather=False, so no
    process group is needed) concatenated in row order equal the whole-domain
    call bit for bit."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import rrtmg, sharding, synthetic
    st = synthetic.make_columns(12, 9, 44, seed=23, fractional_clouds=True)
    for call, kw in ((rrtmg.rrtmg_lwrad_wrf_columns, st.lw_kwargs()), (rrtmg.rrtmg_swrad_wrf_columns, st.sw_kwargs())):
        whole = call(**kw)._asdict()
        slabs = [sharding.sharded_call(call, kw, rank=r, world=2, rows_per_batch=2, gather=False, device=0)
                 for r in range(2)]
        assert slabs[0][0][0] == 0 and slabs[0][0][1] == slabs[1][0][0] and slabs[1][0][1] == 9
        for name, value in whole.items():
            got = np.concatenate([np.asarray(s[1][name]) for s in slabs], axis=-1)
            np.testing.assert_array_equal(got, value, err_msg=name)
