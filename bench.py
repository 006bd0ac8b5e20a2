"""Benchmark: LW+SW radiation columns per second on B200.

Default workload (the metric's own configuration): the learned surrogate with
its per-column gate and plain-kernel fallback on a 1000 x 1000 x 50 domain
(1,000,000 columns, inference generator), against the plain B200 RRTMG
kernels on the same columns.  One step = one full-domain LW+SW radiation
call; `value` is the surrogate+fallback columns/s, `plain_value` the plain
kernels' columns/s, and the line carries the heating and surface-flux RMSE of
the surrogate path against the plain kernels and the fallback fraction.

`--workload plain` measures the plain kernels alone on the 425 x 425 x 50
domain (180,625 columns) with per-launch kernel times and their roofline.

`--workload prologue` measures the radiation prologue (cloud fraction, CAM
ozone, cos zenith) on the 1000 x 1000 x 50 domain against the HBM roofline;
`--workload tendency` the fused radiation tendency chain (LW + SW sum, mass
coupling, accumulation into t_tendf) on 1000 x 51 x 1000 memory arrays.

`e2e` repeats the step with host (numpy) inputs: the host->device copies of
the inputs and the device->host copies of the outputs are inside the timed
region.

On one GPU the default line also carries `ensemble`: the ragged-ensemble
workload (`--workload ensemble`: 12 domains, half surrogate, one CUDA-graph
replay per step against the same domains launched one after another), run in
a child process after the surrogate measurement (`--no-ensemble` leaves it
out).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload surrogate|plain] [--impl reference]

With N > 1 (torchrun, one rank per GPU) every rank runs its own domain (weak
scaling; columns are independent, so there is no collective on the data path)
and the time is the maximum over ranks.

`--impl reference` times the CPU restatement of the reference's algorithm
(oracle/; the reference itself needs jax/jaxlib, which are not installed) on
the host cores, on a bounded sample of the same workload per step.
"""

from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
WORKLOAD = dict(name="plain_425x425x50", nx=425, ny=425, nk=50, seed=0)
SURROGATE_WORKLOAD = dict(name="surrogate_fallback_1000x1000x50", nx=1000, ny=1000, nk=50, seed=2)
WEIGHTS = REPO / "wrf-jax_b200" / "weights" / "surrogate_nk50.npz"
GATE = REPO / "wrf-jax_b200" / "weights" / "surrogate_nk50_gate.json"
METRIC = "LW+SW columns/s on 1 B200: surrogate vs plain RRTMG @ heating RMSE≤0.2 K/day"
# oracle columns timed for the CPU baseline: 100 rows of the domain, about 2-3 s
# on 16 host threads (roughly 40 core-seconds of work)
CPU_SAMPLE_COLUMNS = 42500
# DRAM traffic per unit of the sweep kernels, from ncu (dram__bytes_read.sum +
# dram__bytes_write.sum of one launch divided by its units; the first launch
# on the 256 x 256 x 50 domain, a full chunk): sw_sweep_kernel 15.62 GB over
# 32,768 day columns, lw_sweep_kernel 2.374 GB over 16,384 columns
DRAM_BYTES_PER_DAY_COLUMN_SW = 476700
DRAM_BYTES_PER_COLUMN_LW = 144900
L2_BYTES = 126 * 1024 * 1024
# counted binary32 operations of the plain path per LW column and per SW day
# column (tests/golden/make_flop_counts.py: the oracle's counting build on 10
# rows of the 425 x 425 x 50 generator domain); read as data, nothing under
# oracle/ runs here
FLOP_COUNTS = REPO / "tests" / "golden" / "flop_counts.json"
# FP32 SIMT peak of a B200 (148 SMs x 128 lanes x 2 flops per FMA x 1.965 GHz);
# MEASURED_PEAKS.json has no FP32 figure.  The plain kernels are built without
# FMA contraction (one instruction per add or multiply), so their issue-bound
# ceiling is half of it.
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
# DRAM bytes of one fused-kernel launch per column: dram__bytes_read.sum +
# dram__bytes_write.sum of one mlp_kernel launch on 500,000 columns (ncu, the
# 500 x 1000 x 50 surrogate bench; its 512 MB of feature tiles exceed L2),
# 719,976,960 + 190,990,080 bytes: the reads are the compulsory 1,440 bytes per
# column (feature tile, pi3d, p8w, coszr, flags), the writes just under the
# outputs' 420 (the last ones still in L2 when the kernel ends).  Every byte
# is per column, so a launch's traffic is this times its columns.
MLP_DRAM_BYTES_PER_COLUMN = (719_976_960 + 190_990_080) / 500_000
# compulsory HBM bytes of one column through both calls at nk levels: 12 mass-
# level and 2 interface-level fields read, 4 heating fields written, 37 2-D
# values in or out, binary32
def plain_column_bytes(nk: int) -> int:
    return (18 * nk + 37) * 4


def _package():
    if "wrf_jax_b200" in sys.modules:
        return sys.modules["wrf_jax_b200"]
    root = REPO / "wrf-jax_b200"
    spec = importlib.util.spec_from_file_location(
        "wrf_jax_b200", root / "__init__.py", submodule_search_locations=[str(root)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["wrf_jax_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region.  The sampler
    is started, and its first sample awaited, before the region: nvidia-smi's
    start-up attaches to the driver, which can hold up CUDA calls of other
    processes for a while (the plain bench's enqueues stalled by hundreds of
    ms with the sampler started inside the region).  The first sample, taken
    before the region, is left out of the summary."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device_index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        if self.proc is not None:
            import select
            ready, _, _ = select.select([self.proc.stdout], [], [], 10.0)
            if ready:
                self.proc.stdout.readline()  # the warm-up sample
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]
        else:
            self.lines = []

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_baseline(ncols_sample: int, threads: int | None = None, reps: int = 1, workload: dict | None = None):
    """Time the oracle (CPU restatement, 'port') on a bounded sample of the
    workload: a domain of the workload's row length and generator seed with
    ncols_sample // ny rows."""
    _package()
    from wrf_jax_b200 import synthetic, tables
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle

    wl = workload or WORKLOAD
    threads = threads or os.cpu_count() or 1
    ny = wl["ny"]
    nx = max(1, ncols_sample // ny)
    st = synthetic.make_columns(nx, ny, wl["nk"], seed=wl["seed"])
    kw_lw, kw_sw = st.lw_kwargs(), st.sw_kwargs()
    ora = oracle.Oracle(tables.DEFAULT_BLOB, nthreads=threads)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        ora.lwrad(**kw_lw)
        ora.swrad(**kw_sw)
        times.append(time.perf_counter() - t0)
    cols = nx * ny
    desc = f"{nx}x{ny}x{wl['nk']} columns ({cols}) from the {wl['name']} generator"
    return cols / min(times), threads, desc, min(times)


def run_reference(args, wl: dict):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    sample = int(os.environ.get("RRTMG_CPU_SAMPLE_COLUMNS", str(CPU_SAMPLE_COLUMNS)))
    threads = os.cpu_count() or 1
    times = []
    for _ in range(args.warmup):
        cpu_baseline(sample, threads, workload=wl)
    desc = ""
    for _ in range(args.steps):
        v, th, desc, dt = cpu_baseline(sample, threads, workload=wl)
        times.append(dt)
    dt = statistics.median(times)
    ncols = (sample // wl["ny"]) * wl["ny"]
    value = ncols / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "columns/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
        "config": {"workload": wl["name"], "columns_per_step": ncols, "nk": wl["nk"]},
        "cpu_baseline": {"value": value, "unit": "columns/s", "cores": threads, "kind": "port",
                         "sample": desc + " per step; C restatement of the reference's plain RRTMG path "
                                   "(jax/jaxlib are not installed, so the reference's own JAX code cannot run "
                                   "on this host)"},
        "e2e": {"value": value, "unit": "columns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_plain(args):
    for key in ("nx", "ny", "nk"):
        if getattr(args, key) is not None:
            WORKLOAD[key] = getattr(args, key)
    if any(getattr(args, k) is not None for k in ("nx", "ny", "nk")):
        WORKLOAD["name"] = "plain_%dx%dx%d" % (WORKLOAD["nx"], WORKLOAD["ny"], WORKLOAD["nk"])
    import torch

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    _package()
    from wrf_jax_b200 import _capi, rrtmg, synthetic

    st = synthetic.make_columns(WORKLOAD["nx"], WORKLOAD["ny"], WORKLOAD["nk"], seed=WORKLOAD["seed"] + rank)
    ncol = st.nx * st.ny
    lw_host, sw_host = st.lw_kwargs(), st.sw_kwargs()
    dev = lambda kw: {k: (torch.from_numpy(v).cuda() if isinstance(v, np.ndarray) else v) for k, v in kw.items()}
    lw_dev, sw_dev = dev(lw_host), dev(sw_host)
    ctx = rrtmg.default_context()
    stream = torch.cuda.current_stream()

    def step():
        a = rrtmg.rrtmg_lwrad_wrf_columns(**lw_dev, context=ctx)
        b = rrtmg.rrtmg_swrad_wrf_columns(**sw_dev, context=ctx)
        return a, b

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(max(3, args.warmup)):
        step()
    barrier()
    # per-launch CUDA events recorded by the library on the launching stream
    ctx.check(ctx.lib.rrtmg_timing_enable(ctx.handle, 1))
    # per-call timing (events on the launching stream)
    with ClockSampler(local) as clocks:
        barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        lw_ms, sw_ms = [], []
        t0.record(stream)
        for s in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e2 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rrtmg.rrtmg_lwrad_wrf_columns(**lw_dev, context=ctx)
            e1.record(stream)
            rrtmg.rrtmg_swrad_wrf_columns(**sw_dev, context=ctx)
            e2.record(stream)
            lw_ms.append((e0, e1))
            sw_ms.append((e1, e2))
        t1.record(stream)
        barrier()
    elapsed = t0.elapsed_time(t1) / 1e3
    lw_t = statistics.median(a.elapsed_time(b) for a, b in lw_ms) / 1e3
    sw_t = statistics.median(a.elapsed_time(b) for a, b in sw_ms) / 1e3
    launch_ms = {}
    for side, names in ((0, ("mcica_mask_kernel (LW)", "lw optics (lw_colprep, lw_layer, lw_gas kernels)",
                             "lw_sweep_kernel")),
                        (1, ("mcica_mask_kernel (SW)",
                             "sw optics (sw_daylist, sw_colprep, sw_optics, sw_source kernels)", "sw_sweep_kernel"))):
        buf = (ctypes.c_float * (3 * args.steps))()
        got = ctx.lib.rrtmg_timing_read(ctx.handle, side, buf, args.steps)
        if got != args.steps:
            raise RuntimeError(f"per-launch timing returned {got} calls, expected {args.steps}")
        for k, name in enumerate(names):
            launch_ms[name] = statistics.mean(buf[3 * q + k] for q in range(got))
    ctx.check(ctx.lib.rrtmg_timing_enable(ctx.handle, 0))
    if dist is not None:
        tt = torch.tensor([elapsed], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        elapsed = float(tt.item())
    value = ws * ncol * args.steps / elapsed

    # end-to-end through the public API with host buffers
    # (host inputs in pinned memory, prepared before the timed region; results come back as numpy)
    e2e_steps = max(0, args.e2e_steps) if args.e2e_steps is not None else max(1, min(args.steps, 5))
    pin = lambda kw: {k: (torch.from_numpy(v).pin_memory() if isinstance(v, np.ndarray) else v) for k, v in kw.items()}
    lw_pinned, sw_pinned = pin(lw_host), pin(sw_host)
    h2d = sum(v.nbytes for v in lw_host.values() if isinstance(v, np.ndarray)) + \
        sum(v.nbytes for v in sw_host.values() if isinstance(v, np.ndarray))
    barrier()
    t_e2e = time.perf_counter()
    d2h = 0
    for _ in range(e2e_steps):
        a = rrtmg.rrtmg_lwrad_wrf_columns(**lw_pinned, context=ctx)
        b = rrtmg.rrtmg_swrad_wrf_columns(**sw_pinned, context=ctx)
        d2h = sum(x.nbytes for x in a) + sum(x.nbytes for x in b)
    barrier()
    t_e2e = max(time.perf_counter() - t_e2e, 1e-9)
    if dist is not None:
        tt = torch.tensor([t_e2e], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_e2e = float(tt.item())
    e2e = ws * ncol * e2e_steps / t_e2e

    hbm, bf16, peak_kind = _peaks()
    nk = WORKLOAD["nk"]
    nlay_sw = nk + 1
    sched = _capi.Schedule()
    ctx.check(ctx.lib.rrtmg_get_schedule(ctx.handle, ctypes.byref(sched)))
    lw_chunks = -(-ncol // sched.lw_chunk_columns)
    sw_chunks = -(-ncol // sched.sw_chunk_columns)
    # LW: McICA, then per chunk column set-up, layer set-up, gas optics, sweep;
    # SW: McICA, day list, then per chunk column set-up, layer set-up, band
    # optics, solar source, sweep
    gpu_launches = (1 + 4 * lw_chunks) + (2 + 5 * sw_chunks)
    nday = int((np.asarray(sw_host["coszr"]) > 0.0).sum())
    # The sweep kernels of the staged schedules and their HBM bytes per unit.
    # sw_sweep_kernel, per day column: per layer each g-point's gas and
    # Rayleigh depths and each band's cloud optics from the layer records
    # (2 x 112 + 4 x 14 floats), the clear-sky half of its level stack written
    # and read back (8 floats per level and g-point, twice), the McICA mask (4
    # words per layer), pi3d and p8w for the heating, 2 heating fields and 16
    # 2-D outputs.  The total-sky stack slots, stored only where the g-point
    # layer is cloudy or its total-sky values differ from the clear-sky ones,
    # are data-dependent and not counted: a lower bound on the bytes moved.
    # lw_sweep_kernel, per column: the layer records read in both sweeps
    # (2 x 140 + 4 x 16 + 1 floats per layer, twice), the mask (5 words per
    # layer, twice), pi3d and p8w, 2 heating fields and 15 2-D outputs.
    nlay_lw = ctx.lib.rrtmg_lw_nlayers(float(lw_host["p_top"]), nk)
    unit_bytes = {
        "sw_sweep_kernel": 4 * (nlay_sw * (2 * 112 + 4 * 14) + 2 * 8 * (nlay_sw + 1) * 112 + 4 * nlay_sw
                                + nk + (nk + 1) + 2 * nk + 16),
        "lw_sweep_kernel": 4 * (2 * nlay_lw * (2 * 140 + 4 * 16 + 1) + 2 * 5 * nlay_lw + nk + (nk + 1) + 2 * nk + 15),
    }
    unit_count = {"sw_sweep_kernel": nday, "lw_sweep_kernel": ncol}
    dom = max(("sw_sweep_kernel", "lw_sweep_kernel"), key=lambda k: launch_ms[k])
    units = unit_count[dom]
    dom_s = launch_ms[dom] / 1e3
    achieved = units * unit_bytes[dom] / dom_s / 1e9
    # DRAM bytes per unit measured by ncu (dram__bytes_read.sum +
    # dram__bytes_write.sum of one launch on a smaller case, divided by its units)
    traffic_per_unit = {"sw_sweep_kernel": DRAM_BYTES_PER_DAY_COLUMN_SW, "lw_sweep_kernel": DRAM_BYTES_PER_COLUMN_LW}
    traffic = traffic_per_unit[dom] * units
    plain_fp32 = None
    if FLOP_COUNTS.exists():
        fc = json.loads(FLOP_COUNTS.read_text())
        lw_tf = fc["lw_flops_per_column"] * ncol / lw_t / 1e12
        sw_tf = fc["sw_flops_per_day_column"] * nday / sw_t / 1e12
        plain_fp32 = {"unit": "TFLOP/s", "peak": FP32_PEAK_TFLOPS, "lw_achieved": lw_tf, "lw_frac": lw_tf / FP32_PEAK_TFLOPS,
                      "sw_achieved": sw_tf, "sw_frac": sw_tf / FP32_PEAK_TFLOPS,
                      "flops": "counted binary32 operations per LW column / SW day column: " + fc["sample"]}
    line = {
        "metric": METRIC, "value": value, "unit": "columns/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator; no dataset)",
        "config": {"workload": WORKLOAD["name"], "nx": WORKLOAD["nx"], "ny": WORKLOAD["ny"], "nk": nk,
                   "columns_per_gpu": ncol, "path": "plain RRTMG LW+SW (surrogate not built)",
                   "l2": "inputs larger than L2 (%.0f MB per step)" % (h2d / 1e6),
                   "lw_ms": lw_t * 1e3, "sw_ms": sw_t * 1e3},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "kernel": dom,
                     "kernel_ms": launch_ms[dom], "units_per_launch": units, "bytes_per_unit": unit_bytes[dom],
                     "peak_source": peak_kind,
                     "note": "staged-schedule HBM bytes of the sweep kernel (layer records, level stack, "
                             "mask, I/O) / its time summed over the call's chunks (CUDA events)"},
        "plain_fp32": plain_fp32,
        "launch_ms": launch_ms,
        "gpu_launches": gpu_launches * args.steps,
        "e2e": {"value": e2e, "unit": "columns/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "clocks": clocks.summary(),
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, th, desc, dt = cpu_baseline(int(os.environ.get("RRTMG_CPU_SAMPLE_COLUMNS", str(CPU_SAMPLE_COLUMNS))),
                                       workload=WORKLOAD)
        line["cpu_baseline"] = {"value": v, "unit": "columns/s", "cores": th, "kind": "port", "sample": desc}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def _surrogate_launches(n_fallback: int, fused: bool) -> int:
    """Kernel launches of one surrogate step: features, the fused network
    kernel (or 4 GEMMs and a decode), compact; then the fallback's batched
    gather and scatter, the LW sweep schedule (McICA, column set-up, layer
    set-up, gas optics, sweep) and the SW sweep schedule (McICA, day list,
    column set-up, layer set-up, band optics, solar source, sweep), queued
    with the rejected count left on the device whatever it is; all of the
    fallback once more on a domain of the exact size when more columns are
    rejected than its capacity."""
    from wrf_jax_b200 import surrogate as S
    per_solve = 2 + 5 + 7
    return (3 if fused else 7) + per_solve + (per_solve if n_fallback > S.FALLBACK_CAPACITY else 0)


def run_surrogate(args):
    import torch

    wl = dict(SURROGATE_WORKLOAD)
    if args.nx or args.ny:
        wl["nx"], wl["ny"] = args.nx or wl["nx"], args.ny or wl["ny"]
        wl["name"] = "surrogate_fallback_%dx%dx%d" % (wl["nx"], wl["ny"], wl["nk"])
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    _package()
    from wrf_jax_b200 import surrogate as S, synthetic

    if not WEIGHTS.exists():
        raise FileNotFoundError(f"{WEIGHTS} is missing: train it with wrf-jax_b200/train_surrogate.py")
    model = S.SurrogateModel.load(WEIGHTS)
    tol = json.loads(GATE.read_text())["energy_tol"] if GATE.exists() else 5.0
    st = synthetic.make_columns(wl["nx"], wl["ny"], wl["nk"], seed=wl["seed"] + rank)
    ncol = st.nx * st.ny
    d = S._device_fields(st, "cuda")
    stream = torch.cuda.current_stream()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def timed(fn, steps):
        barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        out = None
        for _ in range(steps):
            out = fn()
        t1.record(stream)
        barrier()
        el = t0.elapsed_time(t1) / 1e3
        if dist is not None:
            tt = torch.tensor([el], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            el = float(tt.item())
        return el, out

    fused = not args.unfused
    sur = lambda: S.infer(model, st, d, energy_tol=tol, fallback=True, fused=fused)
    plain = lambda: S._plain(st, d)
    plain()
    for _ in range(max(3, args.warmup)):
        sur()
    n_plain_steps = max(1, min(args.steps, 3))
    from wrf_jax_b200 import rrtmg
    lw_kw = {k: (d[k] if k in d else v) for k, v in st.lw_kwargs().items()}
    sw_kw = {k: (d[k] if k in d else v) for k, v in st.sw_kwargs().items()}
    with ClockSampler(local) as clocks:
        el_sur, res = timed(sur, args.steps)
        el_plain, (lw, sw) = timed(plain, n_plain_steps)
        el_lw, _ = timed(lambda: rrtmg.rrtmg_lwrad_wrf_columns(**lw_kw), n_plain_steps)
        el_sw, _ = timed(lambda: rrtmg.rrtmg_swrad_wrf_columns(**sw_kw), n_plain_steps)
    value = ws * ncol * args.steps / el_sur
    plain_value = ws * ncol * n_plain_steps / el_plain

    # accuracy of the surrogate path against the plain kernels on the same
    # columns, LW over all columns and SW over the day columns (night SW is
    # exactly zero on both paths)
    pi = d["pi3d"]
    day = (d["coszr"] > 0.0)
    nday = int(day.sum())
    hl, hs = S.heating_kday(res.rthratenlw, pi), S.heating_kday(res.rthratensw, pi)
    rl, rs = S.heating_kday(lw.rthratenlw, pi), S.heating_kday(sw.rthratensw, pi)
    heat_rmse = float(torch.sqrt(torch.cat([(hl - rl).flatten(), (hs - rs).flatten()]).pow(2).mean()))
    flux = torch.stack([res.glw - lw.glw, res.lwupb - lw.lwupb, res.swdnb - sw.swdnb, res.swupb - sw.swupb])
    flux_rmse = float(torch.sqrt((flux ** 2).mean()))
    day3 = day[:, None, :].expand_as(hs)
    accuracy = {
        "lw_heating_rmse_kday": float(torch.sqrt((hl - rl).pow(2).mean())),
        "sw_heating_rmse_kday_day_columns": float(torch.sqrt((hs - rs)[day3].pow(2).mean())),
        "lw_surface_flux_rmse_wm2": float(torch.sqrt(torch.stack([res.glw - lw.glw, res.lwupb - lw.lwupb])
                                                     .pow(2).mean())),
        "sw_surface_flux_rmse_wm2_day_columns": float(torch.sqrt(torch.stack(
            [(res.swdnb - sw.swdnb)[day], (res.swupb - sw.swupb)[day]]).pow(2).mean())),
        "day_columns": nday,
    }

    # the plain kernels against the FP32 SIMT peak, with the counted
    # operations per column, and against the HBM peak with the compulsory bytes
    hbm, bf16, peak_kind = _peaks()
    plain_roofline = None
    if FLOP_COUNTS.exists():
        fc = json.loads(FLOP_COUNTS.read_text())
        lw_ms, sw_ms = el_lw / n_plain_steps * 1e3, el_sw / n_plain_steps * 1e3
        lw_t = fc["lw_flops_per_column"] * ncol / (lw_ms / 1e3) / 1e12
        sw_t = fc["sw_flops_per_day_column"] * nday / (sw_ms / 1e3) / 1e12
        plain_ms = el_plain / n_plain_steps * 1e3
        gbs = plain_column_bytes(wl["nk"]) * ncol / (plain_ms / 1e3) / 1e9
        plain_roofline = {
            "bound": "fp32", "unit": "TFLOP/s", "peak": FP32_PEAK_TFLOPS,
            "peak_source": "nominal FP32 SIMT (148 SMs x 128 lanes x 2 x 1.965 GHz); the path runs without FMA, "
                           "so its issue-bound ceiling is half the peak",
            "lw": {"ms": lw_ms, "flops_per_column": fc["lw_flops_per_column"], "achieved": lw_t,
                   "frac": lw_t / FP32_PEAK_TFLOPS},
            "sw": {"ms": sw_ms, "flops_per_day_column": fc["sw_flops_per_day_column"], "day_columns": nday,
                   "achieved": sw_t, "frac": sw_t / FP32_PEAK_TFLOPS},
            "flop_counts": fc["sample"] + " (" + fc["workload"] + " generator)",
            "hbm": {"bytes_per_column": plain_column_bytes(wl["nk"]), "achieved": gbs, "unit": "GB/s",
                    "peak": hbm, "frac": gbs / hbm,
                    "note": "compulsory I/O of both calls; the staged schedules move their layer records and "
                            "the SW level stack through HBM as well (see profiles/)"},
        }

    # the network alone (the tensor-core part) for the roofline: the fused
    # kernel (four layers + decode), and for comparison the four unfused GEMMs.
    # Algorithmic FLOPs count the network as specified (454 -> 3 x 512 -> 104
    # outputs); the kernel computes padded 512-input and 128-output tiles.
    mpad = (ncol + 127) // 128 * 128
    flops = 2.0 * ncol * (S.N_FEATURES * S.HIDDEN + 2 * S.HIDDEN * S.HIDDEN + S.HIDDEN * 104)
    flops_padded = 2.0 * mpad * sum(o * i for o, i in S.LAYER_SHAPES)
    call = S.fused_kernel_call(model, st, d, energy_tol=tol)
    for _ in range(3):
        call()
    el_fused, _ = timed(call, args.steps)
    fused_ms = el_fused / args.steps * 1e3
    del call
    X = torch.zeros(mpad, S.K_IN, device="cuda", dtype=torch.bfloat16)
    H = [torch.empty(mpad, S.HIDDEN, device="cuda", dtype=torch.bfloat16) for _ in range(3)]
    Y = torch.empty(mpad, S.N_OUT, device="cuda")
    for _ in range(3):
        model.forward(X, H=H, Y=Y)
    el_gemm, _ = timed(lambda: model.forward(X, H=H, Y=Y), args.steps)
    gemm_ms = el_gemm / args.steps * 1e3
    del X, H, Y
    kernel_ms = fused_ms if fused else gemm_ms
    achieved = flops / (kernel_ms / 1e3) / 1e12

    # end to end with host inputs and host outputs through surrogate.infer_host
    # (inputs and outputs in page-locked host memory, allocated before the
    # timed region): the network's fields cross the host link in slabs that
    # overlap the network and the returning outputs; the fallback reads its
    # columns' other inputs from host memory in place (counted below)
    e2e_steps = max(0, args.e2e_steps) if args.e2e_steps is not None else 3
    pinned_in = {k: torch.from_numpy(v).pin_memory() for k, v in st.fields.items()}
    pinned_out = {k: torch.empty(getattr(res, k).shape, pin_memory=True) for k in S.OUTPUT_FIELDS}
    h2d = sum(pinned_in[k].numel() * 4 for k in S.NETWORK_FIELDS)
    d2h = sum(v.numel() * 4 for v in pinned_out.values())
    if e2e_steps:
        n_host = S.infer_host(model, st, pinned_in, pinned_out, energy_tol=tol)  # warm-up
        fb_levels = sum(pinned_in[k].shape[1] if pinned_in[k].dim() == 3 else 1
                        for k in pinned_in if k not in S.NETWORK_FIELDS)
        h2d += n_host * fb_levels * 4  # fallback inputs read in place
        d2h += n_host * (2 * wl["nk"] + 4) * 4  # fallback outputs written in place
    barrier()
    t_e2e = time.perf_counter()
    for _ in range(e2e_steps):
        S.infer_host(model, st, pinned_in, pinned_out, energy_tol=tol)
    barrier()
    t_e2e = max(time.perf_counter() - t_e2e, 1e-9)
    e2e = ws * ncol * e2e_steps / t_e2e if e2e_steps else None

    line = {
        "metric": METRIC, "value": value, "unit": "columns/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el_sur / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (surrogate GEMMs, FP32 accumulate) + f32 (fallback)",
        "data": "synthetic (seeded generator; no dataset)",
        "config": {"workload": wl["name"], "nx": wl["nx"], "ny": wl["ny"], "nk": wl["nk"], "columns_per_gpu": ncol,
                   "l2": "inputs larger than L2 (%.0f MB per step)" % (h2d / 1e6),
                   "energy_gate_tol_wm2": tol, "weights": WEIGHTS.name},
        "plain_value": plain_value, "plain_ms_per_step": el_plain / n_plain_steps * 1e3,
        "speedup_vs_plain": value / plain_value,
        "heating_rmse_kday": heat_rmse, "surface_flux_rmse_wm2": flux_rmse, "accuracy": accuracy,
        "fallback_fraction": res.n_fallback / ncol,
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": bf16, "unit": "TFLOP/s",
                     "frac": achieved / bf16,
                     "traffic": MLP_DRAM_BYTES_PER_COLUMN * ncol if fused else None,
                     "traffic_source": ("ncu DRAM bytes of one launch on 500,000 columns, scaled to the launch's "
                                        "columns" if fused else None),
                     "kernel": "mlp_kernel (4 layers + decode, fused)" if fused else "umma_gemm_kernel (4 GEMMs)",
                     "kernel_ms": kernel_ms, "flops_per_launch": flops, "padded_flops_per_launch": flops_padded,
                     "peak_source": peak_kind, "unfused_gemms_ms": gemm_ms, "fused_ms": fused_ms},
        "plain_roofline": plain_roofline,
        "gpu_launches": _surrogate_launches(res.n_fallback, fused) * args.steps,
        "e2e": {"value": e2e, "unit": "columns/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "clocks": clocks.summary(),
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, th, desc, dt = cpu_baseline(int(os.environ.get("RRTMG_CPU_SAMPLE_COLUMNS", str(CPU_SAMPLE_COLUMNS))),
                                       workload=wl)
        line["cpu_baseline"] = {"value": v, "unit": "columns/s", "cores": th, "kind": "port", "sample": desc}
    if rank == 0 and ws == 1 and not args.no_ensemble:
        line["ensemble"] = ensemble_leg()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


ENSEMBLE_KEYS = ("value", "ms_per_step", "sequential_value", "sequential_ms_per_step", "latency_p50_ms",
                 "latency_p99_ms", "sequential_latency_p50_ms", "sequential_latency_p99_ms", "fallback_columns",
                 "autotune_trials", "clocks")


def ensemble_leg(steps: int = 3, warmup: int = 3, timeout_s: int = 420) -> dict:
    """The ragged-ensemble workload (`--workload ensemble`) run in a child
    process on the same GPU after the surrogate measurement, summarised for the
    default line: graph-replay and sequential columns/s and per-domain
    completion latencies.  A failure is reported in the summary, not raised."""
    cmd = [sys.executable, str(Path(__file__).resolve()), "--workload", "ensemble", "--steps", str(steps),
           "--warmup", str(warmup)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s, cwd=str(REPO))
    except subprocess.TimeoutExpired:
        return {"error": f"ensemble run exceeded {timeout_s} s"}
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    if r.returncode != 0 or not lines:
        tail = (r.stderr or r.stdout).strip().splitlines()[-1:] or [""]
        return {"error": f"ensemble run exited {r.returncode}: {tail[0][:200]}"}
    d = json.loads(lines[-1])
    out = {"workload": d["config"]["workload"], "unit": "columns/s", "columns_per_step": d["config"]["columns_per_step"],
           "schedule": d["config"]["schedule"], "steps": steps, "warmup": warmup}
    out.update({k: d[k] for k in ENSEMBLE_KEYS if k in d})
    return out


def run_ensemble(args):
    """Ragged ensemble (12 domains, U(100,600) x U(100,400) x U{40..60}, half
    surrogate) in one CUDA-graph replay per step against a sequential
    per-domain launch baseline; launch schedule from the project's autotuner."""
    import torch

    _package()
    from wrf_jax_b200 import ensemble as E, surrogate as S

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    model = S.SurrogateModel.load(WEIGHTS)
    tol = json.loads(GATE.read_text())["energy_tol"] if GATE.exists() else 5.0
    members = E.make_members(12, seed=3)
    runner = E.EnsembleRunner(members, model, energy_tol=tol)
    tuned = E.autotune(runner)
    runner.capture()
    for _ in range(max(3, args.warmup)):
        runner.step_graph()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        graph = [runner.step_graph() for _ in range(args.steps)]
        seq = [runner.step_sequential() for _ in range(max(1, min(args.steps, 2)))]
    g_ms = statistics.median(r["ms"] for r in graph)
    s_ms = statistics.median(r["ms"] for r in seq)
    lat_g = [x for r in graph for x in r["latencies_ms"]]
    lat_s = [x for r in seq for x in r["latencies_ms"]]
    ncol = runner.columns
    line = {
        "metric": METRIC, "value": ncol / (g_ms / 1e3), "unit": "columns/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": g_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 (surrogate GEMMs, FP32 accumulate) + f32 (plain, fallback)",
        "data": "synthetic (seeded generator; no dataset)",
        "config": {"workload": "ensemble_12_domains_graph", "domains": [m.name + ":" + m.mode for m in members],
                   "columns_per_step": ncol, "schedule": tuned["best"]},
        "sequential_value": ncol / (s_ms / 1e3), "sequential_ms_per_step": s_ms,
        "latency_p50_ms": E._pct(lat_g, 0.5), "latency_p99_ms": E._pct(lat_g, 0.99),
        "sequential_latency_p50_ms": E._pct(lat_s, 0.5), "sequential_latency_p99_ms": E._pct(lat_s, 0.99),
        "fallback_columns": graph[-1]["fallback_columns"],
        "autotune_trials": len(tuned["trials"]),
        "gpu_launches": None,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)


PROLOGUE_WORKLOAD = dict(name="prologue_1000x1000x50", nx=1000, ny=1000, nk=50, seed=2)


def run_prologue(args):
    """Radiation prologue (cloud fraction, CAM ozone, cos zenith and the
    condensate flag in one launch) on the 1000 x 1000 x 50 inference domain.
    The kernel is HBM-bound: per column it reads qv, qc, qi, qs, t, p (6 nk
    floats) and xlat, xlong, and writes cldfra, o33d (2 nk floats) and coszr:
    (8 nk + 3) * 4 bytes, 1,612 bytes at nk = 50 (the ozone climatology,
    31 KB per block, is served from L2)."""
    import torch

    _package()
    from wrf_jax_b200 import prologue as P, synthetic

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    wl = dict(PROLOGUE_WORKLOAD)
    for k in ("nx", "ny", "nk"):
        if getattr(args, k) is not None:
            wl[k] = getattr(args, k)
            wl["name"] = f"prologue_{wl['nx']}x{wl['ny']}x{wl['nk']}"
    nx, ny, nk = wl["nx"], wl["ny"], wl["nk"]
    st = synthetic.make_columns(nx=nx, ny=ny, nk=nk, seed=wl["seed"] + rank)
    xlat, xlong = synthetic.lat_lon(nx, ny, seed=wl["seed"] + rank)
    names = ("qv3d", "qc3d", "qi3d", "qs3d", "t3d", "p3d")
    host = {k: torch.from_numpy(st.fields[k]).pin_memory() for k in names}
    host["xlat"] = torch.from_numpy(xlat).pin_memory()
    host["xlong"] = torch.from_numpy(xlong).pin_memory()
    dev = {k: v.cuda() for k, v in host.items()}
    plev, lat, oz = synthetic.cam_ozone_climatology(seed=0)
    P.set_ozone_climatology(plev * np.float32(100.0), lat, oz)
    outs = {"cldfra3d": torch.empty((nx, nk, ny), device="cuda"), "o33d": torch.empty((nx, nk, ny), device="cuda"),
            "coszr": torch.empty((nx, ny), device="cuda"),
            "condensate_present": torch.empty((), dtype=torch.int32, device="cuda")}
    kw = dict(julian=172.3, xtime=195.0, gmt=6.0, yr=2019, radt=30.0, case_dir=False)

    def step(src):
        return P.radiation_prologue(qv=src["qv3d"], qc=src["qc3d"], qi=src["qi3d"], qs=src["qs3d"], t3d=src["t3d"],
                                    p3d=src["p3d"], xlat=src["xlat"], xlong=src["xlong"], out=outs, **kw)

    for _ in range(max(3, args.warmup)):
        step(dev)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for a, b in ev:   # inputs (1.2 GB) exceed L2: no flush needed between steps
            a.record()
            step(dev)
            b.record()
        t1.record()
        torch.cuda.synchronize()
    total_ms = t0.elapsed_time(t1)
    kernel_ms = statistics.median(a.elapsed_time(b) for a, b in ev)
    if ws > 1:
        t = torch.tensor([total_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    ms = total_ms / args.steps
    ncol = nx * ny
    # end to end: pinned host inputs copied in, outputs copied back, every step
    h_out = {k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True) for k, v in outs.items()}
    h2d = sum(v.numel() * 4 for v in host.values())
    d2h = sum(v.numel() * v.element_size() for v in outs.values())
    e2e_steps = args.e2e_steps or max(2, min(args.steps, 5))
    for _ in range(2):
        step({k: v.cuda(non_blocking=True) for k, v in host.items()})
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(e2e_steps):
        step({k: v.cuda(non_blocking=True) for k, v in host.items()})
        for k, v in outs.items():
            h_out[k].copy_(v, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    hbm, _, src = _peaks()
    alg = (8 * nk + 3) * 4 * ncol
    achieved = alg / (kernel_ms * 1e-3) / 1e9
    line = {
        "metric": "radiation prologue columns/s on 1 B200 (cloud fraction, CAM ozone, cos zenith)",
        "value": ncol * ws / (ms / 1e3), "unit": "columns/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator; CAM ozone stand-in)",
        "config": {"workload": wl["name"], "nx": nx, "ny": ny, "nk": nk, "columns_per_gpu": ncol,
                   "l2": "inputs (1.2 GB) larger than L2"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "peak_source": src, "kernel": "prologue_kernel",
                     "algorithmic_bytes_per_column": (8 * nk + 3) * 4, "kernel_ms": kernel_ms},
        "e2e": {"value": ncol / (e2e_ms / 1e3), "unit": "columns/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": 2 * args.steps,  # condensate-flag reset + the prologue kernel
        "clocks": clocks.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, str(REPO / "oracle"))
        import prologue_oracle as PO
        rows = 64
        sub = {k: st.fields[k][:rows] for k in names}
        t = time.perf_counter()
        declin, _ = PO.radconst(172.3)
        PO.cal_cldfra1(*(sub[k] for k in names))
        PO.cam_o3rad(xlat[:rows], sub["p3d"], julian=172.3, plev=plev * np.float32(100.0), lat_oz=lat, ozone=oz)
        PO.calc_coszen(xlat[:rows], xlong[:rows], julian=172.3, xtime=210.0, gmt=6.0, declin=declin)
        dt = time.perf_counter() - t
        line["cpu_baseline"] = {"value": rows * ny / dt, "unit": "columns/s", "cores": 1, "kind": "port",
                                "sample": f"{rows} x {ny} x {nk} columns through the numpy oracle"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()


def run_tendency(args):
    """Radiation tendency chain (LW + SW heating, mass coupling over the tile,
    accumulation into t_tendf) in one pass over a 1000 x 51 x 1000 memory
    domain (WRF mass arrays: 50 levels plus the unused top slot), tile = the
    whole domain.  HBM-bound: per element it reads rthratenlw, rthratensw and
    rt_tendf and writes rthraten, and rt_tendf on the tile's levels (20 bytes,
    16 on the unused top slot)."""
    import torch

    _package()
    from wrf_jax_b200 import tendency as TD

    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    nx = args.nx or 1000
    ny = args.ny or 1000
    nk = (args.nk or 50) + 1
    b = dict(ids=1, ide=nx + 1, jds=1, jde=ny + 1, kds=1, kde=nk, ims=1, ime=nx, jms=1, jme=ny, kms=1, kme=nk,
             its=1, ite=nx, jts=1, jte=ny, kts=1, kte=nk - 1)
    tb = TD.bounds({}, **b)
    rng = np.random.default_rng(5 + rank)
    shape = (nx, nk, ny)
    host = {
        "lw": torch.from_numpy(rng.normal(-2e-5, 1e-5, shape).astype(np.float32)).pin_memory(),
        "sw": torch.from_numpy(rng.normal(1e-5, 1e-5, shape).astype(np.float32)).pin_memory(),
        "t": torch.from_numpy(rng.normal(0, 3, shape).astype(np.float32)).pin_memory(),
    }
    c1 = torch.from_numpy(rng.uniform(0, 1, nk).astype(np.float32)).cuda()
    c2 = torch.from_numpy(rng.uniform(0, 5000, nk).astype(np.float32)).cuda()
    mut = torch.from_numpy(rng.uniform(5e4, 9.5e4, (nx, ny)).astype(np.float32)).cuda()
    dev = {k: v.cuda() for k, v in host.items()}
    r = torch.empty(shape, device="cuda")
    from wrf_jax_b200 import _capi
    lib = _capi.load()

    def step(src):
        st = lib.rrtmg_radiation_tendency(ctypes.byref(tb), src["lw"].data_ptr(), src["sw"].data_ptr(),
                                          c1.data_ptr(), c2.data_ptr(), mut.data_ptr(), 1, r.data_ptr(),
                                          src["t"].data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        if st != 0:
            raise RuntimeError(f"rrtmg_radiation_tendency failed: {st}")

    for _ in range(max(3, args.warmup)):
        step(dev)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for a, b_ in ev:   # 1 GB of arrays per step: larger than L2
            a.record()
            step(dev)
            b_.record()
        t1.record()
        torch.cuda.synchronize()
    total_ms = t0.elapsed_time(t1)
    kernel_ms = statistics.median(a.elapsed_time(b_) for a, b_ in ev)
    if ws > 1:
        tt = torch.tensor([total_ms], device="cuda")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(tt.item())
    ms = total_ms / args.steps
    ncol = nx * ny
    h_r = torch.empty(shape, pin_memory=True)
    h_t = torch.empty(shape, pin_memory=True)
    e2e_steps = args.e2e_steps or max(2, min(args.steps, 5))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(e2e_steps):
        step({k: v.cuda(non_blocking=True) for k, v in host.items()})
        h_r.copy_(r, non_blocking=True)
        h_t.copy_(dev["t"], non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    hbm, _, src = _peaks()
    # reads lw, sw, rt_tendf and writes rthraten everywhere; rt_tendf is written
    # back on the tile's levels only (kts..kde-1: not the unused top slot)
    alg = nx * ny * (16 * nk + 4 * (nk - 1))
    achieved = alg / (kernel_ms * 1e-3) / 1e9
    line = {
        "metric": "radiation tendency columns/s on 1 B200 (LW+SW sum, mass coupling, t_tendf accumulation)",
        "value": ncol * ws / (ms / 1e3), "unit": "columns/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"tendency_{nx}x{nk}x{ny}", "memory_levels": nk, "columns_per_gpu": ncol,
                   "l2": "arrays (1 GB) larger than L2"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "peak_source": src,
                     "kernel": "tendency_kernel_vec4" if ny % 4 == 0 else "tendency_kernel",
                     "algorithmic_bytes_per_column": 16 * nk + 4 * (nk - 1), "kernel_ms": kernel_ms},
        "e2e": {"value": ncol / (e2e_ms / 1e3), "unit": "columns/s", "h2d_bytes_per_step": 3 * 4 * nx * nk * ny,
                "d2h_bytes_per_step": 2 * 4 * nx * nk * ny},
        "gpu_launches": args.steps,
        "clocks": clocks.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, str(REPO / "oracle"))
        import tendency_oracle as TO
        rows = 100
        bb = dict(b, ime=rows, ite=rows, ide=rows + 1)
        lw, sw, tt = (host[k].numpy()[:rows] for k in ("lw", "sw", "t"))
        t = time.perf_counter()
        TO.radiation_tendency(lw, sw, c1.cpu().numpy(), c2.cpu().numpy(), mut.cpu().numpy()[:rows], tt, bb)
        dt = time.perf_counter() - t
        line["cpu_baseline"] = {"value": rows * ny / dt, "unit": "columns/s", "cores": 1, "kind": "port",
                                "sample": f"{rows} x {nk} x {ny} through the numpy oracle"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--workload", choices=("surrogate", "plain", "ensemble", "prologue", "tendency"), default="surrogate")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nx", type=int, default=None, help="override the plain domain (profiling cases)")
    ap.add_argument("--ny", type=int, default=None)
    ap.add_argument("--nk", type=int, default=None)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--unfused", action="store_true", help="surrogate network as 4 GEMMs + decode kernel")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="leave out the ragged-ensemble leg of the default line (profiling runs)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args, SURROGATE_WORKLOAD if args.workload == "surrogate" else WORKLOAD)
    elif args.workload == "plain":
        run_plain(args)
    elif args.workload == "ensemble":
        run_ensemble(args)
    elif args.workload == "prologue":
        run_prologue(args)
    elif args.workload == "tendency":
        run_tendency(args)
    else:
        run_surrogate(args)


if __name__ == "__main__":
    main()
