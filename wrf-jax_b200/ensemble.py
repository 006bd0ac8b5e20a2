"""Ragged ensemble of radiation domains in one CUDA-graph replay.

An ensemble is a set of domains with different grid sizes and level counts
(seeded U(100, 600) x U(100, 400) columns x U{40..60} levels).  Half of them use
the plain kernels and half the surrogate (whose domains have the network's 50
levels).  All launches of one ensemble step (plain LW/SW calls, surrogate
features, forward GEMMs and decode) are captured once into a CUDA graph over
several streams, so independent domains overlap on the GPU, and replayed with
one launch per step.  The columns the surrogate's gate rejects, from every
surrogate domain, are then gathered into one compact domain and solved by one
plain LW + SW call (one fallback per step instead of one per domain).

`autotune` picks the launch schedule (columns per launch of the plain kernels,
the band-split limit of the SW kernel, the GEMM tile width, the number of
streams) by timing candidate settings on the ensemble itself.
"""

from __future__ import annotations

import ctypes
import json
import math
import statistics
from dataclasses import dataclass, field

import numpy as np

from . import _capi, rrtmg, surrogate as S, synthetic


# cost of a plain column in surrogate columns (the surrogate path runs about
# 150 times more columns per second than the plain kernels)
PLAIN_COST = 150.0


@dataclass
class Member:
    name: str
    mode: str                      # "plain" or "surrogate"
    st: object                     # synthetic.ColumnState
    d: dict = field(default_factory=dict)     # device inputs
    out: dict = field(default_factory=dict)   # device outputs
    buf: dict = field(default_factory=dict)   # surrogate buffers

    @property
    def columns(self) -> int:
        return self.st.nx * self.st.ny


def make_members(n: int = 12, seed: int = 3) -> list[Member]:
    """The ensemble of the survey's config 4: grids U(100, 600) x U(100, 400),
    U{40..60} levels; even members plain, odd members surrogate (50 levels)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    members = []
    for i in range(n):
        nx = int(rng.integers(100, 601))
        ny = int(rng.integers(100, 401))
        nk = int(rng.integers(40, 61))
        mode = "plain" if i % 2 == 0 else "surrogate"
        if mode == "surrogate":
            nk = S.NK
        st = synthetic.make_columns(nx, ny, nk, seed=seed * 1000 + i)
        members.append(Member(name=f"d{i:02d}_{nx}x{ny}x{nk}", mode=mode, st=st))
    return members


class EnsembleRunner:
    def __init__(self, members: list[Member], model: S.SurrogateModel, *, energy_tol: float = 5.0,
                 streams: int = 4):
        import torch

        self.members = members
        self.model = model
        self.energy_tol = energy_tol
        self.ctx = rrtmg.default_context()
        self.graph = None
        self.set_streams(streams)
        self.stamps = torch.zeros(len(members) + 2, device="cuda", dtype=torch.int64)
        for m in members:
            m.d = {k: torch.from_numpy(v).cuda() for k, v in m.st.fields.items()}
            nx, ny, nk = m.st.nx, m.st.ny, m.st.nk
            if m.mode == "plain":
                m.out["lw"] = {k: torch.empty((nx, nk, ny) if k.startswith("rthraten") else (nx, ny), device="cuda")
                               for k in _capi.LW_OUT_FIELDS}
                m.out["sw"] = {k: torch.empty((nx, nk, ny) if k.startswith("rthraten") else (nx, ny), device="cuda")
                               for k in _capi.SW_OUT_FIELDS}
            else:
                ncol = nx * ny
                mpad = (ncol + 127) // 128 * 128
                m.buf = dict(X=torch.zeros(mpad, S.K_IN, device="cuda", dtype=torch.bfloat16),
                             flags=torch.empty(ncol, device="cuda", dtype=torch.int32),
                             list=torch.empty(ncol, device="cuda", dtype=torch.int32),
                             count=torch.zeros(1, device="cuda", dtype=torch.int32))
                m.out = {"rthratenlw": torch.empty(nx, nk, ny, device="cuda"),
                         "rthratensw": torch.empty(nx, nk, ny, device="cuda")}
                for k in ("glw", "lwupb", "swdnb", "swupb"):
                    m.out[k] = torch.empty(nx, ny, device="cuda")
                # the member's own fallback domain (its count stays on the
                # device, so the fallback is captured with the member)
                lw_kw, sw_kw = m.st.lw_kwargs(), m.st.sw_kwargs()
                m.buf["plan"] = S._FallbackPlan(
                    nk, min(ncol, S.FALLBACK_CAPACITY),
                    {k: lw_kw[k] for k in S._SCALAR_KEYS_LW if k in lw_kw},
                    {k: sw_kw[k] for k in S._SCALAR_KEYS_SW if k in sw_kw})

    def set_streams(self, n: int) -> None:
        import torch
        self.streams = [torch.cuda.Stream() for _ in range(max(1, n))]
        self.graph = None

    @property
    def columns(self) -> int:
        return sum(m.columns for m in self.members)

    # -- launches -----------------------------------------------------------------
    def _launch_member(self, m: Member, stream, fallback: bool = False) -> None:
        """Queue one member on `stream`; fallback: also the surrogate member's
        own re-solve of the columns its gate rejects, with the count left on
        the device (up to the member's fallback capacity)."""
        lib = _capi.load()
        sid = stream.cuda_stream
        if m.mode == "plain":
            lw_kw = {k: (m.d[k] if k in m.d else v) for k, v in m.st.lw_kwargs().items()}
            sw_kw = {k: (m.d[k] if k in m.d else v) for k, v in m.st.sw_kwargs().items()}
            rrtmg.rrtmg_lwrad_wrf_columns(**lw_kw, context=self.ctx, stream=sid, out=m.out["lw"])
            rrtmg.rrtmg_swrad_wrf_columns(**sw_kw, context=self.ctx, stream=sid, out=m.out["sw"])
            return
        st, b = m.st, m.buf
        s = ctypes.c_void_p(sid)
        # features in the tile layout, then the fused network and gated decode
        S._network(self.model, m.d, st.nx, st.ny, st.nk, m.out, b["flags"], self.energy_tol, b["X"], s)
        b["count"].zero_()
        S._check(lib.rrtmg_sur_compact(b["flags"].data_ptr(), m.columns, b["list"].data_ptr(),
                                       b["count"].data_ptr(), s), "compact")
        if fallback:
            S._solve_listed(b["plan"], lib, s, b["list"], b["count"], st.ny, m.d, m.out, None, live=True)

    def launch_order(self) -> list[int]:
        """Members cheapest first (shortest processing time first minimises the
        mean completion time on one stream; with several streams the cheap
        members finish while the expensive ones run).  Cost: columns, a plain
        column weighted as PLAIN_COST surrogate columns."""
        cost = [m.columns * (PLAIN_COST if m.mode == "plain" else 1.0) for m in self.members]
        return sorted(range(len(self.members)), key=lambda i: cost[i])

    def _stamp(self, slot: int, stream) -> None:
        lib = _capi.load()
        S._check(lib.rrtmg_sur_timestamp(self.stamps[slot:].data_ptr(), ctypes.c_void_p(stream.cuda_stream)),
                 "timestamp")

    def launch_all(self, stamp: bool = False, fallback: bool = False) -> None:
        """Every launch of one step, spread over the streams (fork from and
        join to the current stream); fallback: each surrogate member's own
        device-counted fallback too (else the merged fallback runs after).
        With stamp, the GPU timer is written at the start (slot 0) and after
        each domain (slot i+1)."""
        import torch
        main = torch.cuda.current_stream()
        if stamp:
            self._stamp(0, main)
        fork = torch.cuda.Event()
        fork.record(main)
        order = self.launch_order()
        for q, i in enumerate(order):
            s = self.streams[q % len(self.streams)]
            s.wait_event(fork)
            with torch.cuda.stream(s):
                self._launch_member(self.members[i], s, fallback=fallback)
                if stamp:
                    self._stamp(i + 1, s)
        for s in self.streams:
            join = torch.cuda.Event()
            join.record(s)
            main.wait_event(join)

    def merged_fallback(self) -> int:
        """Solve the rejected columns of every surrogate domain in one plain call."""
        import torch
        lib = _capi.load()
        sur = [m for m in self.members if m.mode == "surrogate"]
        if not sur:
            return 0
        counts = torch.cat([m.buf["count"] for m in sur]).cpu().tolist()
        total = int(sum(counts))
        if total == 0:
            return 0
        s = torch.cuda.current_stream().cuda_stream
        nk = S.NK
        sub = {k: torch.empty(1, nk, total, device="cuda") for k in S._FIELDS_3D}
        sub.update({k: torch.empty(1, nk + 1, total, device="cuda") for k in S._FIELDS_LEV})
        sub.update({k: torch.empty(1, total, device="cuda") for k in S._FIELDS_2D})

        nz = {k: nk for k in S._FIELDS_3D}
        nz.update({k: nk + 1 for k in S._FIELDS_LEV})
        nz.update({k: 1 for k in S._FIELDS_2D})

        def move(m, pairs, to, off, n):
            f = _capi.SurFields(nfields=len(pairs))
            for i, (src, dst, z) in enumerate(pairs):
                f.src[i], f.dst[i], f.nz[i] = src.data_ptr(), dst.data_ptr(), z
            S._check(lib.rrtmg_sur_move_fields(m.buf["list"].data_ptr(), m.buf["count"].data_ptr(), n, m.st.ny,
                                               ctypes.byref(f), to, total, off, ctypes.c_void_p(s)), "move fields")

        off = 0
        for m, n in zip(sur, counts):
            if n:
                move(m, [(m.d[k], sub[k], z) for k, z in nz.items()], 1, off, n)
            off += n
        ref = sur[0].st  # scalars (gases, solar constant, flags) are common to the generator's domains
        lw_kw = {k: (sub[k] if k in sub else v) for k, v in ref.lw_kwargs().items()}
        sw_kw = {k: (sub[k] if k in sub else v) for k, v in ref.sw_kwargs().items()}
        lw = rrtmg.rrtmg_lwrad_wrf_columns(**lw_kw, context=self.ctx)
        sw = rrtmg.rrtmg_swrad_wrf_columns(**sw_kw, context=self.ctx)
        off = 0
        for m, n in zip(sur, counts):
            if n:
                move(m, [(lw.rthratenlw, m.out["rthratenlw"], nk), (sw.rthratensw, m.out["rthratensw"], nk),
                         (lw.glw, m.out["glw"], 1), (lw.lwupb, m.out["lwupb"], 1), (sw.swdnb, m.out["swdnb"], 1),
                         (sw.swupb, m.out["swupb"], 1)], 0, off, n)
            off += n
        return total

    # -- graph --------------------------------------------------------------------
    def capture(self) -> None:
        """Warm up (table jumps, pools, kernel attributes), then capture one
        step: every member, each surrogate member's fallback included."""
        import torch
        for _ in range(2):
            self.launch_all(fallback=True)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.launch_all(stamp=True, fallback=True)
        torch.cuda.synchronize()

    def step_graph(self) -> dict:
        """One replayed step; per-domain completion times (ms from the step
        start, fallbacks included) and the step time.  A surrogate member
        whose gate rejected more columns than its fallback capacity has them
        all re-solved after the replay (on an exact-size domain), and its
        completion is the end of that."""
        import torch
        if self.graph is None:
            self.capture()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        self.graph.replay()
        counts = [int(m.buf["count"].item()) if m.mode == "surrogate" else 0 for m in self.members]
        over = [m for m, n in zip(self.members, counts) if m.mode == "surrogate" and n > m.buf["plan"].cap]
        for m in over:
            saved = self.members
            self.members = [m]
            self.merged_fallback()
            self.members = saved
        self._stamp(len(self.members) + 1, torch.cuda.current_stream())
        end.record()
        torch.cuda.synchronize()
        total = start.elapsed_time(end)
        ts = self.stamps.cpu().tolist()
        t0, t_end = ts[0], ts[len(self.members) + 1]
        lat = [((t_end if m in over else ts[i + 1]) - t0) / 1e6 for i, m in enumerate(self.members)]
        return dict(ms=total, latencies_ms=lat, fallback_columns=sum(counts))

    def step_sequential(self) -> dict:
        """The baseline: one domain after another in the members' order, each
        launched and finished (its own fallback included) before the next
        starts.  A domain's latency is its completion time since the step
        started, as for the graph step."""
        import torch
        lat = []
        main = torch.cuda.current_stream()
        t0 = torch.cuda.Event(enable_timing=True)
        t0.record()
        n_fb = 0
        for m in self.members:
            b = torch.cuda.Event(enable_timing=True)
            self._launch_member(m, main)
            if m.mode == "surrogate":
                saved = self.members
                self.members = [m]
                n_fb += self.merged_fallback()
                self.members = saved
            b.record()
            torch.cuda.synchronize()
            lat.append(t0.elapsed_time(b))
        t1 = torch.cuda.Event(enable_timing=True)
        t1.record()
        torch.cuda.synchronize()
        return dict(ms=t0.elapsed_time(t1), latencies_ms=lat, fallback_columns=n_fb)


def _pct(values, q: float) -> float:
    v = sorted(values)
    if not v:
        return float("nan")
    k = (len(v) - 1) * q
    lo, hi = math.floor(k), math.ceil(k)
    return v[lo] + (v[hi] - v[lo]) * (k - lo)


def summarize(runner: EnsembleRunner, result: dict) -> dict:
    return dict(columns=runner.columns, ms=result["ms"], columns_per_s=runner.columns / (result["ms"] / 1e3),
                latency_p50_ms=_pct(result["latencies_ms"], 0.5), latency_p99_ms=_pct(result["latencies_ms"], 0.99),
                fallback_columns=result["fallback_columns"])


def autotune(runner: EnsembleRunner, *, log=None) -> dict:
    """Coordinate search over the launch schedule, timing sequential steps of
    the ensemble (the schedule is fixed once a graph is captured)."""
    import torch
    lib = _capi.load()
    ctx = runner.ctx

    def apply(cfg):
        sch = _capi.Schedule(lw_chunk_columns=cfg["lw_chunk"], sw_chunk_columns=cfg["sw_chunk"],
                             sw_split_max_columns=cfg["sw_split_max"], lw_split_max_columns=cfg["lw_split_max"])
        ctx.check(lib.rrtmg_set_schedule(ctx.handle, ctypes.byref(sch)))
        S._check(lib.rrtmg_gemm_set_tile(cfg["gemm_tile"]), "gemm tile")
        runner.set_streams(cfg["streams"])

    def measure(cfg):
        apply(cfg)
        runner.launch_all(fallback=True)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(2):
            runner.launch_all(fallback=True)
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / 2

    space = dict(lw_chunk=[65536, 131072, 262144], sw_chunk=[65536, 131072, 262144],
                 sw_split_max=[2048, 4096, 8192], lw_split_max=[1024, 2048, 4096], gemm_tile=[128, 256],
                 streams=[1, 2, 4])
    best = dict(lw_chunk=131072, sw_chunk=131072, sw_split_max=4096, lw_split_max=2048, gemm_tile=256, streams=4)
    best_ms = measure(best)
    trials = [dict(best, ms=best_ms)]
    for key, values in space.items():
        for v in values:
            if v == best[key]:
                continue
            cand = dict(best, **{key: v})
            ms = measure(cand)
            trials.append(dict(cand, ms=ms))
            if log:
                log(f"autotune {key}={v}: {ms:.2f} ms (best {best_ms:.2f})")
            if ms < best_ms:
                best, best_ms = cand, ms
    best, best_ms = prefer_fewer_streams(best, best_ms, trials)
    apply(best)
    return dict(best=best, best_ms=best_ms, trials=trials)


def prefer_fewer_streams(best: dict, best_ms: float, trials: list, tol: float = 0.01) -> tuple:
    """Among the trials that differ from `best` only in the stream count, the
    one with the fewest streams whose step time is within `tol` of the best.
    On fewer streams the members run closer to their cheapest-first order, so
    most of them complete early (median per-domain completion 7 ms on one
    stream against 54 ms on four for the 12-domain ensemble, at under 1% of
    throughput).  Returns (schedule, step ms)."""
    same = [t for t in trials if all(t.get(k) == v for k, v in best.items() if k != "streams")]
    same.append(dict(best, ms=best_ms))
    ok = [t for t in same if t["ms"] <= best_ms * (1.0 + tol)]
    pick = min(ok, key=lambda t: (t["streams"], t["ms"]))
    return {k: pick[k] for k in best}, pick["ms"]
