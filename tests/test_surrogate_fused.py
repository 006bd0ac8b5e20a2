"""Fused surrogate inference (rrtmg_sur_mlp: four tcgen05 layers and the
decode in one kernel) against the unfused path (one GEMM per layer, then
rrtmg_sur_decode).  Both compute the same operations in the same order, so
the bar is bit-for-bit equality of every output field and gate flag; the
layouts the fused kernel reads (feature tiles, packed weights) are checked
element for element against the row-major matrices."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

WEIGHTS = REPO / "wrf-jax_b200" / "weights" / "surrogate_nk50.npz"


@pytest.fixture(scope="module")
def torch_cuda(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def model(torch_cuda):
    from wrf_jax_b200 import surrogate as S
    return S.SurrogateModel.load(WEIGHTS)


def _unswizzle(img: np.ndarray, blocks: int, rows: int) -> np.ndarray:
    """[blocks, rows, 64] BF16 (as uint16) from blocks of the 128-byte swizzled
    K-major layout: chunk kc of row r sits at chunk position kc ^ (r & 7)."""
    v = img.reshape(blocks, rows, 8, 8)
    r = np.arange(rows)[:, None]
    kc = np.arange(8)[None, :]
    return v[:, r, kc ^ (r & 7), :].reshape(blocks, rows, 64)


def _features(torch, model, st, d, x_layout, old_kernel=False):
    from wrf_jax_b200 import _capi, surrogate as S
    lib = _capi.load()
    ncol = st.nx * st.ny
    mpad = (ncol + 127) // 128 * 128
    X = torch.zeros(mpad, S.K_IN, device="cuda", dtype=torch.bfloat16)
    flags = torch.full((ncol,), 7, device="cuda", dtype=torch.int32)
    fa = S._feature_args(d, st.nk, st.ny, ncol)
    fa.mean, fa.rstd = model.norm.in_mean.data_ptr(), model.norm.in_rstd.data_ptr()
    fa.X, fa.ldx, fa.x_layout = X.data_ptr(), S.K_IN, x_layout
    fa.lo, fa.hi, fa.flags = model.norm.in_lo.data_ptr(), model.norm.in_hi.data_ptr(), flags.data_ptr()
    Xt = None
    if old_kernel:  # a transposed copy is only written by the tiled shared-memory kernel
        Xt = torch.zeros(S.K_IN, ncol, device="cuda", dtype=torch.bfloat16)
        fa.Xt, fa.ldxt = Xt.data_ptr(), ncol
    assert lib.rrtmg_sur_features(ctypes.byref(fa), torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    return X, flags


@pytest.mark.parametrize("nx,ny", [(37, 29), (64, 50), (40, 36), (17, 64), (6, 1000)])
def test_feature_layouts_match_the_reference_kernel(torch_cuda, model, nx, ny):
    """Warps of 32 columns that straddle west-east rows (ny = 29, 36, 50,
    1000) or fall on row starts (ny = 64), and a partial last warp."""
    torch = torch_cuda
    from wrf_jax_b200 import surrogate as S, synthetic
    st = synthetic.make_columns(nx, ny, S.NK, seed=21)
    d = S._device_fields(st, "cuda")
    ncol = nx * ny
    X_old, f_old = _features(torch, model, st, d, 0, old_kernel=True)
    X_row, f_row = _features(torch, model, st, d, 0)
    X_tile, f_tile = _features(torch, model, st, d, 1)
    a = X_old.view(torch.int16).cpu().numpy()[:ncol]
    assert np.array_equal(X_row.view(torch.int16).cpu().numpy()[:ncol], a)
    tiles = X_tile.view(torch.int16).cpu().numpy().view(np.uint16).reshape(-1, 8, 128 * 64)
    T = tiles.shape[0]
    un = _unswizzle(tiles.reshape(T * 8, 128 * 64), T * 8, 128).reshape(T, 8, 128, 64)
    rowmajor = un.transpose(0, 2, 1, 3).reshape(T * 128, 512)[:ncol]
    assert np.array_equal(rowmajor, a.view(np.uint16))
    assert torch.equal(f_row, f_old) and torch.equal(f_tile, f_old)


def test_packed_weight_image(torch_cuda, model):
    torch = torch_cuda
    from wrf_jax_b200 import _capi
    img = model.weight_image().cpu().numpy().view(np.uint16)
    assert img.size * 2 == _capi.WEIGHT_IMAGE_BYTES
    hidden = img[:48 * 16384].reshape(48, 256 * 64)
    un = _unswizzle(hidden, 48, 256).reshape(3, 2, 8, 256, 64)
    for layer in range(3):
        w = model.wb[layer].view(torch.int16).cpu().numpy().view(np.uint16)
        got = un[layer].transpose(0, 2, 1, 3).reshape(512, 512)
        assert np.array_equal(got, w), layer
    last = _unswizzle(img[48 * 16384:].reshape(8, 128 * 64), 8, 128)
    w3 = model.wb[3].view(torch.int16).cpu().numpy().view(np.uint16)
    assert np.array_equal(last.transpose(1, 0, 2).reshape(128, 512), w3)


@pytest.mark.parametrize("nx,ny", [(9, 7), (96, 70), (200, 150)])
def test_fused_inference_equals_unfused(torch_cuda, model, nx, ny):
    """9 x 7: one partial tile; 96 x 70: a ragged last tile; 200 x 150: more
    tiles than SMs, so CTAs loop over several tiles."""
    torch = torch_cuda
    from wrf_jax_b200 import surrogate as S, synthetic
    S.gemm_error(reset=True)
    st = synthetic.make_columns(nx, ny, S.NK, seed=33)
    d = S._device_fields(st, "cuda")
    ref = S.infer(model, st, d, energy_tol=5.0, fallback=False, fused=False)
    for _ in range(2):  # the second call reuses the workspace
        got = S.infer(model, st, d, energy_tol=5.0, fallback=False, fused=True)
        torch.cuda.synchronize()
        assert S.gemm_error() == 0
        for name in ("rthratenlw", "rthratensw", "glw", "lwupb", "swdnb", "swupb", "flags"):
            a, b = getattr(ref, name), getattr(got, name)
            assert torch.equal(a, b), (name, float((a.float() - b.float()).abs().max()))


def test_fused_inference_with_fallback_matches_plain_bits_on_rejected_columns(torch_cuda, model):
    torch = torch_cuda
    from wrf_jax_b200 import surrogate as S, synthetic
    st = synthetic.make_columns(64, 48, S.NK, seed=5)
    d = S._device_fields(st, "cuda")
    res = S.infer(model, st, d, energy_tol=1.0, fallback=True, fused=True)
    lw, sw = S._plain(st, d)
    torch.cuda.synchronize()
    rej = (res.flags != 0).view(st.nx, st.ny)
    assert res.n_fallback == int(rej.sum()) and res.n_fallback > 0
    m3 = rej[:, None, :].expand(st.nx, st.nk, st.ny)
    assert torch.equal(res.rthratenlw[m3], lw.rthratenlw[m3])
    assert torch.equal(res.rthratensw[m3], sw.rthratensw[m3])
    assert torch.equal(res.glw[rej], lw.glw[rej]) and torch.equal(res.swdnb[rej], sw.swdnb[rej])


def test_fused_rejects_other_level_counts(torch_cuda, model):
    torch = torch_cuda
    from wrf_jax_b200 import _capi
    lib = _capi.load()
    a = _capi.SurMlpArgs(ncol=128, nk=40, ny=8)
    assert lib.rrtmg_sur_mlp(ctypes.byref(a), None) == 1


def test_infer_host_equals_device_path(torch_cuda, model):
    """Host-buffer pipeline (slabs over the host link, fallback reading and
    writing host memory in place) against infer() on device fields: the same
    bits, including the fallback columns (a tight energy gate rejects many)."""
    torch = torch_cuda
    from wrf_jax_b200 import surrogate as S, synthetic
    st = synthetic.make_columns(40, 36, S.NK, seed=9)
    d = S._device_fields(st, "cuda")
    ref = S.infer(model, st, d, energy_tol=1.0, fallback=True)
    torch.cuda.synchronize()
    host = {k: torch.from_numpy(v).pin_memory() for k, v in st.fields.items()}
    out = {k: torch.empty(tuple(getattr(ref, k).shape), pin_memory=True) for k in S.OUTPUT_FIELDS}
    for slabs in (8, 3, 1):  # 8: tapered last slabs (6 x 6 rows, then 3 and 1)
        for t in out.values():
            t.fill_(float("nan"))
        n = S.infer_host(model, st, host, out, energy_tol=1.0, slabs=slabs)
        assert n == ref.n_fallback and n > 0
        for k in S.OUTPUT_FIELDS:
            assert torch.equal(out[k], getattr(ref, k).cpu()), k


def test_fallback_overflow_takes_the_exact_size_pass(torch_cuda, model):
    """More rejected columns than the sync-free capacity: every one of them
    still carries the plain kernels' bits."""
    torch = torch_cuda
    from wrf_jax_b200 import surrogate as S, synthetic
    st = synthetic.make_columns(100, 100, S.NK, seed=8)
    d = S._device_fields(st, "cuda")
    res = S.infer(model, st, d, energy_tol=0.5, fallback=True)
    lw, sw = S._plain(st, d)
    torch.cuda.synchronize()
    assert res.n_fallback > S.FALLBACK_CAPACITY
    rej = (res.flags != 0).view(st.nx, st.ny)
    assert int(rej.sum()) == res.n_fallback
    m3 = rej[:, None, :].expand(st.nx, st.nk, st.ny)
    assert torch.equal(res.rthratenlw[m3], lw.rthratenlw[m3])
    assert torch.equal(res.rthratensw[m3], sw.rthratensw[m3])
    assert torch.equal(res.lwupb[rej], lw.lwupb[rej]) and torch.equal(res.swupb[rej], sw.swupb[rej])


def test_live_count_calls_match_full_calls(torch_cuda):
    """rrtmg_lwrad_live / rrtmg_swrad_live with a device count below the
    domain size: the counted columns equal the full call's, the others keep
    what the output buffers held."""
    torch = torch_cuda
    from wrf_jax_b200 import _capi, rrtmg, surrogate as S, synthetic
    st = synthetic.make_columns(1, 300, 47, seed=12)
    d = S._device_fields(st, "cuda")
    lw_ref, sw_ref = S._plain(st, d)
    ctx = rrtmg.default_context()
    live = torch.tensor([173], device="cuda", dtype=torch.int32)
    lw_kw, sw_kw = st.lw_kwargs(), st.sw_kwargs()
    scal = lambda kw, keys: {k: kw[k] for k in keys if k in kw}
    cfg_lw = rrtmg.lw_config(1, 300, 47, **scal(lw_kw, S._SCALAR_KEYS_LW))
    cfg_sw = rrtmg.sw_config(1, 300, 47, **scal(sw_kw, S._SCALAR_KEYS_SW))
    lw_out = {k: torch.full(tuple(getattr(lw_ref, k).shape), -7.0, device="cuda") for k in _capi.LW_OUT_FIELDS}
    sw_out = {k: torch.full(tuple(getattr(sw_ref, k).shape), -7.0, device="cuda") for k in _capi.SW_OUT_FIELDS}
    s = torch.cuda.current_stream().cuda_stream
    ctx.check(ctx.lib.rrtmg_lwrad_live(ctx.handle, ctypes.byref(cfg_lw),
                                       ctypes.byref(_capi.LwIn(**{k: d[k].data_ptr() for k in _capi.LW_IN_FIELDS})),
                                       ctypes.byref(_capi.LwOut(**{k: v.data_ptr() for k, v in lw_out.items()})),
                                       ctypes.c_void_p(live.data_ptr()), ctypes.c_void_p(s)))
    ctx.check(ctx.lib.rrtmg_swrad_live(ctx.handle, ctypes.byref(cfg_sw),
                                       ctypes.byref(_capi.SwIn(**{k: d[k].data_ptr() for k in _capi.SW_IN_FIELDS})),
                                       ctypes.byref(_capi.SwOut(**{k: v.data_ptr() for k, v in sw_out.items()})),
                                       ctypes.c_void_p(live.data_ptr()), ctypes.c_void_p(s)))
    torch.cuda.synchronize()
    for name, ref, got in [(k, getattr(lw_ref, k), lw_out[k]) for k in _capi.LW_OUT_FIELDS] + \
                          [(k, getattr(sw_ref, k), sw_out[k]) for k in _capi.SW_OUT_FIELDS]:
        if got.dim() == 3:
            assert torch.equal(got[:, :, :173], ref[:, :, :173]), name
            assert bool((got[:, :, 173:] == -7.0).all()), name
        else:
            assert torch.equal(got[:, :173], ref[:, :173]), name
            assert bool((got[:, 173:] == -7.0).all()), name
    # a host pointer is refused before anything runs
    host_count = ctypes.c_int(5)
    st_code = ctx.lib.rrtmg_lwrad_live(ctx.handle, ctypes.byref(cfg_lw),
                                       ctypes.byref(_capi.LwIn(**{k: d[k].data_ptr() for k in _capi.LW_IN_FIELDS})),
                                       ctypes.byref(_capi.LwOut(**{k: v.data_ptr() for k, v in lw_out.items()})),
                                       ctypes.cast(ctypes.byref(host_count), ctypes.c_void_p), ctypes.c_void_p(s))
    assert st_code == 1
