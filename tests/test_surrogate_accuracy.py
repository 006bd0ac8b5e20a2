"""The committed surrogate (wrf-jax_b200/weights/surrogate_nk50.npz) on a
held-out 256 x 256 x 50 domain of the inference generator (seed 7: training
used seed 1 with widened perturbations, the gate calibration seed 3 and the
benchmark seed 2), with its gate and plain-kernel fallback, against the plain
kernels on the same columns.

Bars: the specified heating RMSE <= 0.2 K/day and surface-flux RMSE
<= 2 W/m2 over LW and SW together (every column), with at most 5 % of the
columns sent to the fallback.  Each side alone is held to 0.2 K/day too (SW
over the day columns only: night SW is exactly zero on both paths).  The SW
surface fluxes over the day columns alone come to about 2.05 W/m2 on this
domain (the pooled figure includes the exact zeros of the night columns and
the smaller LW errors), so their bar is 2.5 W/m2, and the value is printed.
"""

from __future__ import annotations

import json

import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

WEIGHTS = REPO / "wrf-jax_b200" / "weights" / "surrogate_nk50.npz"
GATE = REPO / "wrf-jax_b200" / "weights" / "surrogate_nk50_gate.json"


def test_held_out_domain_meets_accuracy_targets(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import surrogate as S, synthetic

    model = S.SurrogateModel.load(WEIGHTS)
    tol = json.loads(GATE.read_text())["energy_tol"]
    st = synthetic.make_columns(256, 256, S.NK, seed=7)
    d = S._device_fields(st, "cuda")
    res = S.infer(model, st, d, energy_tol=tol, fallback=True)
    lw, sw = S._plain(st, d)
    pi = d["pi3d"]
    day = d["coszr"] > 0.0
    day3 = day[:, None, :].expand(-1, S.NK, -1)
    hl, rl = S.heating_kday(res.rthratenlw, pi), S.heating_kday(lw.rthratenlw, pi)
    hs, rs = S.heating_kday(res.rthratensw, pi), S.heating_kday(sw.rthratensw, pi)
    rmse = lambda x: float(torch.sqrt((x.double() ** 2).mean()))
    heat_all = rmse(torch.cat([(hl - rl).flatten(), (hs - rs).flatten()]))
    heat_lw = rmse(hl - rl)
    heat_sw_day = rmse((hs - rs)[day3])
    flux_all = rmse(torch.stack([res.glw - lw.glw, res.lwupb - lw.lwupb, res.swdnb - sw.swdnb,
                                 res.swupb - sw.swupb]))
    flux_lw = rmse(torch.stack([res.glw - lw.glw, res.lwupb - lw.lwupb]))
    flux_sw_day = rmse(torch.stack([(res.swdnb - sw.swdnb)[day], (res.swupb - sw.swupb)[day]]))
    ncol = st.nx * st.ny
    print(f"\nheld-out 256x256: heating RMSE {heat_all:.4f} K/day (LW {heat_lw:.4f}, SW day {heat_sw_day:.4f}); "
          f"surface flux RMSE {flux_all:.3f} W/m2 (LW {flux_lw:.3f}, SW day {flux_sw_day:.3f}); "
          f"fallback {res.n_fallback}/{ncol}")
    assert heat_all <= 0.2 and heat_lw <= 0.2 and heat_sw_day <= 0.2
    assert flux_all <= 2.0 and flux_lw <= 2.0 and flux_sw_day <= 2.5
    assert res.n_fallback <= 0.05 * ncol
    # the fallback columns carry the plain kernels' bits
    if res.n_fallback:
        idx = torch.nonzero(res.flags.view(st.nx, st.ny) != 0)
        i, j = idx[:, 0], idx[:, 1]
        assert torch.equal(res.rthratenlw[i, :, j], lw.rthratenlw[i, :, j])
        assert torch.equal(res.rthratensw[i, :, j], sw.rthratensw[i, :, j])
