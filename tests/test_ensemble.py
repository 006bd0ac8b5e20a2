"""Ragged ensemble in one CUDA-graph replay: outputs equal those of the same
calls made one by one (plain domains bit for bit against rrtmg_*rad; surrogate
domains against surrogate.infer)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_graph_ensemble_matches_direct_calls(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import ensemble as E, rrtmg, surrogate as S, synthetic
    from conftest import REPO

    model = S.SurrogateModel.load(REPO / "wrf-jax_b200" / "weights" / "surrogate_nk50.npz")
    members = [E.Member("p0", "plain", synthetic.make_columns(120, 90, 44, seed=1)),
               E.Member("s1", "surrogate", synthetic.make_columns(96, 80, S.NK, seed=2)),
               E.Member("p2", "plain", synthetic.make_columns(100, 110, 57, seed=3))]
    runner = E.EnsembleRunner(members, model, energy_tol=1.0, streams=2)
    runner.capture()
    res = runner.step_graph()
    assert len(res["latencies_ms"]) == 3
    for m in members:
        if m.mode == "plain":
            lw = rrtmg.rrtmg_lwrad_wrf_columns(**m.st.lw_kwargs())
            sw = rrtmg.rrtmg_swrad_wrf_columns(**m.st.sw_kwargs())
            for name in lw._fields:
                np.testing.assert_array_equal(m.out["lw"][name].cpu().numpy(), getattr(lw, name), err_msg=name)
            for name in sw._fields:
                np.testing.assert_array_equal(m.out["sw"][name].cpu().numpy(), getattr(sw, name), err_msg=name)
        else:
            ref = S.infer(model, m.st, energy_tol=1.0, fallback=True)
            assert res["fallback_columns"] == ref.n_fallback
            for name in ("rthratenlw", "rthratensw", "glw", "lwupb", "swdnb", "swupb"):
                np.testing.assert_array_equal(m.out[name].cpu().numpy(), getattr(ref, name).cpu().numpy(),
                                              err_msg=name)
