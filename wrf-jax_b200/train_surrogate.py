"""Train the radiation surrogate on the GPU and evaluate it against the plain
kernels (run from the repository root):

    python wrf-jax_b200/train_surrogate.py --columns 2000000 --epochs 30 \\
        --out wrf-jax_b200/weights/surrogate_nk50.npz

Training data: columns from the seeded generator with widened perturbations
(T noise N(0, 4 K), RH U(0.05, 1), cloud probability U(0, 0.6) per column),
solved by the plain B200 RRTMG kernels.  Evaluation: a held-out domain from the
default generator (inference configuration), surrogate with gate and fallback
against the plain kernels on the same columns.
"""

from __future__ import annotations

import argparse
import importlib.util
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _package():
    if "wrf_jax_b200" in sys.modules:
        return sys.modules["wrf_jax_b200"]
    spec = importlib.util.spec_from_file_location("wrf_jax_b200", HERE / "__init__.py",
                                                  submodule_search_locations=[str(HERE)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["wrf_jax_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def evaluate(model, nx: int, ny: int, seed: int, energy_tol: float) -> dict:
    """Surrogate (with and without fallback) against the plain kernels on one domain."""
    import torch
    from wrf_jax_b200 import surrogate as S, synthetic

    st = synthetic.make_columns(nx, ny, S.NK, seed=seed)
    d = S._device_fields(st, "cuda")
    lw, sw = S._plain(st, d)
    pi = d["pi3d"]
    ref_lw = S.heating_kday(lw.rthratenlw, pi)
    ref_sw = S.heating_kday(sw.rthratensw, pi)
    out = {}
    for tag, fb in (("surrogate_only", False), ("with_fallback", True)):
        res = S.infer(model, st, d, energy_tol=energy_tol, fallback=fb)
        hl = S.heating_kday(res.rthratenlw, pi)
        hs = S.heating_kday(res.rthratensw, pi)
        day = (d["coszr"] > 0).reshape(nx, 1, ny).expand_as(hs)
        rm = lambda a, b: float(torch.sqrt(((a - b) ** 2).mean()))
        flux = torch.stack([res.glw - lw.glw, res.lwupb - lw.lwupb, res.swdnb - sw.swdnb, res.swupb - sw.swupb])
        out[tag] = dict(
            heating_rmse_kday=float(torch.sqrt(torch.cat([(hl - ref_lw).flatten(), (hs - ref_sw).flatten()]).pow(2)
                                               .mean())),
            lw_heating_rmse_kday=rm(hl, ref_lw),
            sw_heating_rmse_kday=rm(hs, ref_sw),
            sw_heating_rmse_day_kday=float(torch.sqrt(((hs - ref_sw)[day] ** 2).mean())),
            surface_flux_rmse_wm2=float(torch.sqrt((flux ** 2).mean())),
            fallback_columns=int(res.n_fallback),
            flagged_fraction=float((res.flags != 0).float().mean()),
            flagged_range=int((res.flags & 1).ne(0).sum()),
            flagged_energy=int((res.flags & 2).ne(0).sum()),
        )
    return out


def calibrate_gate(model, nx: int, ny: int, seed: int, heating_target: float = 0.2, flux_target: float = 2.0,
                   tolerances=(1e30, 20.0, 10.0, 5.0, 3.0, 2.0, 1.5, 1.0, 0.75, 0.5, 0.3, 0.2, 0.1, 0.05),
                   max_tol: float = 5.0) -> dict:
    """Energy-gate tolerance sweep on a calibration domain: the largest
    tolerance up to max_tol whose surrogate+fallback heating and surface-flux
    RMSE against the plain kernels meet the targets (0: every column falls
    back).  The ceiling keeps the energy-consistency check active; the sweep
    still records the larger tolerances (1e30: no energy check)."""
    import torch
    from wrf_jax_b200 import surrogate as S, synthetic

    st = synthetic.make_columns(nx, ny, S.NK, seed=seed)
    d = S._device_fields(st, "cuda")
    lw, sw = S._plain(st, d)
    pi = d["pi3d"]
    rl, rs = S.heating_kday(lw.rthratenlw, pi), S.heating_kday(sw.rthratensw, pi)
    sweep, chosen = [], 0.0
    for tol in tolerances:
        res = S.infer(model, st, d, energy_tol=tol, fallback=True)
        hl, hs = S.heating_kday(res.rthratenlw, pi), S.heating_kday(res.rthratensw, pi)
        heat = float(torch.sqrt(torch.cat([(hl - rl).flatten(), (hs - rs).flatten()]).pow(2).mean()))
        flux = torch.stack([res.glw - lw.glw, res.lwupb - lw.lwupb, res.swdnb - sw.swdnb, res.swupb - sw.swupb])
        fl = float(torch.sqrt((flux ** 2).mean()))
        frac = res.n_fallback / (nx * ny)
        sweep.append(dict(energy_tol=tol, heating_rmse_kday=heat, surface_flux_rmse_wm2=fl, fallback_fraction=frac))
        if heat <= heating_target and fl <= flux_target and chosen == 0.0 and tol <= max_tol:
            chosen = tol
    return dict(energy_tol=chosen, heating_target_kday=heating_target, flux_target_wm2=flux_target,
                calibration_domain=[nx, ny, seed], sweep=sweep, max_energy_tol=max_tol)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--columns", type=int, default=2_000_000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--energy-tol", type=float, default=5.0)
    ap.add_argument("--eval", type=int, nargs=2, default=(256, 256), metavar=("NX", "NY"))
    ap.add_argument("--out", type=Path, required=True)
    ap.add_argument("--metrics", type=Path, default=None)
    ap.add_argument("--gate", type=Path, default=None, help="write the calibrated energy-gate tolerance here")
    args = ap.parse_args(argv)
    _package()
    import torch
    from wrf_jax_b200 import surrogate as S

    t0 = time.time()
    raw, T = S.generate_dataset(args.columns, seed=args.seed)
    torch.cuda.synchronize()
    t_data = time.time() - t0
    model = S.SurrogateModel(seed=args.seed)
    model.fit_normalization(raw, T)
    X, Tn = model.normalized(raw, T)
    del raw, T
    torch.cuda.synchronize()
    t1 = time.time()
    hist = S.train(model, X, Tn, epochs=args.epochs, batch=args.batch, lr=args.lr, seed=args.seed)
    torch.cuda.synchronize()
    t_train = time.time() - t1
    flag = S.gemm_error()
    args.out.parent.mkdir(parents=True, exist_ok=True)
    model.save(args.out)
    metrics = dict(columns=args.columns, epochs=args.epochs, batch=args.batch, lr=args.lr, seed=args.seed,
                   data_seconds=t_data, train_seconds=t_train, steps=model.step, loss_history=hist,
                   gemm_timeout_flag=flag,
                   eval=evaluate(model, args.eval[0], args.eval[1], seed=2, energy_tol=args.energy_tol))
    gate = calibrate_gate(model, 256, 256, seed=3)
    metrics["gate"] = gate
    metrics["eval_calibrated"] = evaluate(model, args.eval[0], args.eval[1], seed=2, energy_tol=gate["energy_tol"])
    if args.gate:
        args.gate.write_text(json.dumps(gate, indent=1))
    text = json.dumps(metrics, indent=1)
    print(text)
    if args.metrics:
        args.metrics.write_text(text)
    return 0 if flag == 0 else 1


if __name__ == "__main__":
    raise SystemExit(main())
