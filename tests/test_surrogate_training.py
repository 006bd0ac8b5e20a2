"""Surrogate training kernels on the GPU: gradients of one training step
against the CPU oracle (oracle/surrogate_oracle.py), and a short training run
showing what the trained network gains over the untrained one (its
climatological mean).  The trained network's accuracy against the plain
kernels is tests/test_surrogate_accuracy.py; its speed is bench.py's
surrogate line."""

from __future__ import annotations

import sys

import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_training_step_gradients_match_cpu_oracle(torch_cuda):
    """Tolerance: relative Frobenius error 2e-2 per gradient (BF16 activations
    may round one ulp apart between erff on the GPU and erf in float64)."""
    torch = torch_cuda
    sys.path.insert(0, str(REPO / "oracle"))
    import surrogate_oracle as so
    from wrf_jax_b200 import surrogate as S

    B = 512
    model = S.SurrogateModel(seed=3)
    g = torch.Generator(device="cuda").manual_seed(7)
    X = (torch.randn(B, S.K_IN, device="cuda", generator=g)).bfloat16()
    X[:, S.N_FEATURES:] = 0
    Tn = torch.randn(B, S.N_OUT, device="cuda", generator=g)
    w = S.target_weights()
    idx = torch.arange(B, device="cuda", dtype=torch.int32)
    wb = [x.float().cpu().numpy() for x in model.wb]
    bs = [x.cpu().numpy() for x in model.b]
    model.train_step(X, Tn, idx, w, lr=0.0)
    torch.cuda.synchronize()
    assert S.gemm_error() == 0
    buf = model._buf
    _, gw, gb = so.forward_backward(X.float().cpu().numpy(), Tn.cpu().numpy(), wb, bs, w.cpu().numpy(),
                                    1.0 / (B * S.N_TARGETS))
    for layer in range(4):
        got_w = buf["gw"][layer].cpu().numpy()
        got_b = buf["gb"][layer].cpu().numpy()
        ew = np.linalg.norm(got_w - gw[layer]) / max(np.linalg.norm(gw[layer]), 1e-30)
        eb = np.linalg.norm(got_b - gb[layer]) / max(np.linalg.norm(gb[layer]), 1e-30)
        assert ew < 2e-2, (layer, ew)
        assert eb < 2e-2, (layer, eb)


def test_short_training_beats_untrained_network(torch_cuda):
    torch = torch_cuda
    from wrf_jax_b200 import surrogate as S, synthetic

    raw, T = S.generate_dataset(131072, seed=11, log=None)
    model = S.SurrogateModel(seed=0)
    model.fit_normalization(raw, T)
    X, Tn = model.normalized(raw, T)
    hist = S.train(model, X, Tn, epochs=4, batch=16384, lr=2e-3, log=None)
    assert hist[-1] < 0.7 * hist[0]
    # held-out domain: trained network against the climatological mean (untrained output 0)
    st = synthetic.make_columns(128, 128, S.NK, seed=12345, t_noise=4.0, rh_lo=0.05, cloud_p=(0.0, 0.6))
    res = S.infer(model, st, fallback=False)
    raw_t, T_t = S.generate_dataset(128 * 128, seed=12345, chunk=(128, 128), log=None)
    _, Tn_t = model.normalized(raw_t, T_t)
    Xt_, _ = model.normalized(raw_t, T_t)
    Y = model.forward(Xt_, H=[torch.empty(Xt_.shape[0], S.HIDDEN, device="cuda", dtype=torch.bfloat16)
                              for _ in range(3)])
    mse_trained = float(((Y[:, :S.N_TARGETS] - Tn_t[:, :S.N_TARGETS]) ** 2).mean())
    mse_mean = float((Tn_t[:, :S.N_TARGETS] ** 2).mean())
    assert mse_trained < 0.5 * mse_mean
    assert res.flags.shape[0] == 128 * 128
