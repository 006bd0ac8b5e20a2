"""Learned radiation surrogate: an MLP from a column profile to LW/SW heating
profiles and surface fluxes, trained and run on B200 tensor cores.

Network: 454 inputs (9 per-level fields x 50 levels + 4 surface scalars,
zero-padded to 512) -> 3 hidden layers of 512 with GELU -> 106 outputs (50 LW
and 50 SW heating rates [K/day], 4 surface fluxes, and 2 gate-only outputs: the
LW and SW net fluxes at the model top), padded to 128.  Weights are BF16 for
the tensor cores with an FP32 Adam master copy; all GEMMs are the hand-written
tcgen05 kernel of librrtmg_b200.so (FP32 accumulation in tensor memory), and
every other arithmetic step (features, targets, normalization, batch gather,
loss gradient, bias gradients, split-K sums, Adam, decode, gate, fallback
gather/scatter) is a CUDA kernel of the same library.  torch only holds device
buffers and the stream.

Inference with fallback: every column is predicted; a column is rejected when
an input lies outside the training range or when its predicted heating does
not integrate to its predicted net-flux divergence (energy gate).  Rejected
columns are gathered into a compact domain, solved by the plain RRTMG kernels,
and scattered back, so their outputs are the plain kernel's bits.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _capi

NK = 50                    # model levels the network is built for
N_FEATURES = 9 * NK + 4    # 454
N_TARGETS = 2 * NK + 6     # 106
K_IN = 512                 # padded input width
N_OUT = 128                # padded output width
HIDDEN = 512
LAYER_SHAPES = ((HIDDEN, K_IN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (N_OUT, HIDDEN))  # (out, in)
HEATFAC = (9.8066 * 8.6400e4) / (1004.5 * 1.0e2)


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def _stream(stream=None) -> ctypes.c_void_p:
    import torch
    return ctypes.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)


def _check(st: int, what: str) -> None:
    if st != 0:
        raise RuntimeError(f"{what} failed with status {st}")


def gemm_bf16(A, B, *, epilogue: int = _capi.EPI_F32, bias=None, C=None, ksplit: int = 1, H=None, Ht=None,
              aux=None, Z=None, stream=None) -> None:
    """C[M x N] = A[M x K] @ B[N x K]^T on the tensor cores, with the epilogue
    of include/rrtmg_surrogate.h.  A and B are contiguous bf16 CUDA tensors;
    outputs are preallocated tensors (C: float32 [ksplit, M, N] or [M, N];
    H: bf16 [M, N]; Ht: bf16 [N, M]; Z, aux: float32 [M, N])."""
    M, K = A.shape
    N, K2 = B.shape
    if K2 != K:
        raise ValueError(f"inner dimensions differ: {K} vs {K2}")
    lib = _capi.load()
    g = _capi.GemmArgs()
    g.A, g.lda, g.B, g.ldb = A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0)
    g.M, g.N, g.K, g.ksplit, g.epilogue = M, N, K, ksplit, epilogue
    g.bias = _ptr(bias)
    if C is not None:
        g.C, g.ldc = C.data_ptr(), C.stride(-2)
        g.split_stride = C.stride(0) if C.dim() == 3 else 0
    if H is not None:
        g.H, g.ldh = H.data_ptr(), H.stride(0)
    if Ht is not None:
        g.Ht, g.ldht = Ht.data_ptr(), Ht.stride(0)
    if aux is not None:
        g.aux, g.ldaux = aux.data_ptr(), aux.stride(0)
    if Z is not None:
        g.Z, g.ldz = Z.data_ptr(), Z.stride(0)
    st = lib.rrtmg_gemm_bf16(ctypes.byref(g), _stream(stream))
    if st != 0:
        raise ValueError(f"rrtmg_gemm_bf16 rejected the arguments (status {st}): M={M} N={N} K={K} ksplit={ksplit}")


def gemm_error(reset: bool = True) -> int:
    """Synchronous read of the GEMM timeout flag (0 = no CTA gave up; the call
    itself reports a set flag as RRTMG_TIMEOUT, returned here as the flag)."""
    flag = ctypes.c_uint(0)
    st = _capi.load().rrtmg_gemm_error(int(reset), ctypes.byref(flag))
    if st not in (0, 4):  # RRTMG_OK, RRTMG_TIMEOUT
        _check(st, "rrtmg_gemm_error")
    return flag.value


# ---------------------------------------------------------------------------
# features and targets
# ---------------------------------------------------------------------------
def _feature_args(d: dict, nk: int, ny: int, ncol: int, row_offset: int = 0) -> _capi.SurFeaturesArgs:
    a = _capi.SurFeaturesArgs()
    a.ncol, a.nk, a.ny, a.row_offset = ncol, nk, ny, row_offset
    a.p3d, a.p8w, a.t3d = _ptr(d["p3d"]), _ptr(d["p8w"]), _ptr(d["t3d"])
    a.qv, a.qc, a.qi, a.qs = _ptr(d["qv3d"]), _ptr(d["qc3d"]), _ptr(d["qi3d"]), _ptr(d["qs3d"])
    a.cldfra, a.o3, a.tsk = _ptr(d["cldfra3d"]), _ptr(d["o33d"]), _ptr(d["tsk"])
    a.albedo, a.coszr, a.emiss = _ptr(d["albedo"]), _ptr(d["coszr"]), _ptr(d["emiss"])
    return a


def _device_fields(st, device: str) -> dict:
    import torch
    return {k: torch.from_numpy(v).to(device) for k, v in st.fields.items()}


def _plain(st, d: dict):
    from . import rrtmg
    lw_kw = {k: (d[k] if k in d else v) for k, v in st.lw_kwargs().items()}
    sw_kw = {k: (d[k] if k in d else v) for k, v in st.sw_kwargs().items()}
    return rrtmg.rrtmg_lwrad_wrf_columns(**lw_kw), rrtmg.rrtmg_swrad_wrf_columns(**sw_kw)


def generate_dataset(n_columns: int, *, seed: int = 1, chunk: tuple[int, int] = (512, 256), t_noise: float = 4.0,
                     rh_lo: float = 0.05, cloud_p=(0.0, 0.6), log=print):
    """Columns from the seeded generator (widened perturbations), solved by the
    plain B200 kernels.  Returns raw FP32 features [n, N_FEATURES] and targets
    [n, N_OUT] on the GPU."""
    import torch
    from . import synthetic

    lib = _capi.load()
    cx, cy = chunk
    per = cx * cy
    nchunks = math.ceil(n_columns / per)
    n = nchunks * per
    raw = torch.empty(n, N_FEATURES, device="cuda")
    T = torch.empty(n, N_OUT, device="cuda")
    for q in range(nchunks):
        st = synthetic.make_columns(cx, cy, NK, seed=seed * 1000 + q, t_noise=t_noise, rh_lo=rh_lo, cloud_p=cloud_p)
        d = _device_fields(st, "cuda")
        lw, sw = _plain(st, d)
        fa = _feature_args(d, NK, cy, per, q * per)
        fa.raw, fa.ldf = raw.data_ptr(), raw.stride(0)
        _check(lib.rrtmg_sur_features(ctypes.byref(fa), _stream()), "rrtmg_sur_features")
        ta = _capi.SurTargetsArgs()
        ta.ncol, ta.nk, ta.ny, ta.row_offset = per, NK, cy, q * per
        ta.rthratenlw, ta.rthratensw = lw.rthratenlw.data_ptr(), sw.rthratensw.data_ptr()
        ta.pi3d, ta.p8w = d["pi3d"].data_ptr(), d["p8w"].data_ptr()
        ta.glw, ta.lwupb = lw.glw.data_ptr(), lw.lwupb.data_ptr()
        ta.swdnb, ta.swupb = sw.swdnb.data_ptr(), sw.swupb.data_ptr()
        ta.T, ta.ldt = T.data_ptr(), T.stride(0)
        _check(lib.rrtmg_sur_targets(ctypes.byref(ta), _stream()), "rrtmg_sur_targets")
        if log and (q % 4 == 0 or q == nchunks - 1):
            torch.cuda.synchronize()
            log(f"dataset chunk {q + 1}/{nchunks}")
    torch.cuda.synchronize()
    return raw[:n_columns], T[:n_columns]


# ---------------------------------------------------------------------------
# model
# ---------------------------------------------------------------------------
@dataclass
class Normalization:
    in_mean: object
    in_rstd: object
    in_lo: object
    in_hi: object
    out_mean: object
    out_std: object


class SurrogateModel:
    """Weights (FP32 master + BF16 copies), Adam moments and normalization, on one GPU."""

    def __init__(self, seed: int = 0):
        import torch

        rng = np.random.Generator(np.random.PCG64(seed))
        self.w, self.b = [], []
        for out_f, in_f in LAYER_SHAPES:
            w = rng.normal(0.0, 1.0 / math.sqrt(in_f), size=(out_f, in_f)).astype(np.float32)
            self.w.append(torch.from_numpy(w).cuda())
            self.b.append(torch.zeros(out_f, device="cuda"))
        if LAYER_SHAPES[0][1] > N_FEATURES:  # padded inputs carry no weight
            self.w[0][:, N_FEATURES:] = 0.0
        self.wb = [w.to(torch.bfloat16).contiguous() for w in self.w]
        self.wbt = [w.t().contiguous().to(torch.bfloat16) for w in self.w]
        self.mw = [torch.zeros_like(w) for w in self.w]
        self.vw = [torch.zeros_like(w) for w in self.w]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.step = 0
        self.norm: Normalization | None = None

    # -- normalization ------------------------------------------------------
    def fit_normalization(self, raw, T) -> None:
        import torch
        lib = _capi.load()
        f = lambda n: torch.zeros(n, device="cuda")
        in_mean, in_rstd, in_lo, in_hi = f(K_IN), f(K_IN), f(K_IN), f(K_IN)
        _check(lib.rrtmg_sur_column_stats(raw.data_ptr(), raw.shape[0], raw.stride(0), N_FEATURES,
                                          in_mean.data_ptr(), in_rstd.data_ptr(), in_lo.data_ptr(),
                                          in_hi.data_ptr(), _stream()), "column stats (inputs)")
        out_mean, out_rstd = f(N_OUT), f(N_OUT)
        _check(lib.rrtmg_sur_column_stats(T.data_ptr(), T.shape[0], T.stride(0), N_TARGETS, out_mean.data_ptr(),
                                          out_rstd.data_ptr(), None, None, _stream()), "column stats (targets)")
        torch.cuda.synchronize()
        # outputs: a constant target (rstd 0) keeps std 1; widened input range for the gate
        out_std = torch.where(out_rstd > 0, 1.0 / torch.where(out_rstd > 0, out_rstd, torch.ones_like(out_rstd)),
                              torch.ones_like(out_rstd))
        span = (in_hi - in_lo) * 0.05
        self.norm = Normalization(in_mean, in_rstd, in_lo - span, in_hi + span, out_mean, out_std)

    def normalized(self, raw, T):
        """BF16 normalized inputs [n, K_IN] and FP32 normalized targets [n, N_OUT]."""
        import torch
        lib = _capi.load()
        n = raw.shape[0]
        X = torch.empty(n, K_IN, device="cuda", dtype=torch.bfloat16)
        _check(lib.rrtmg_sur_normalize(raw.data_ptr(), raw.stride(0), n, N_FEATURES, self.norm.in_mean.data_ptr(),
                                       self.norm.in_rstd.data_ptr(), X.data_ptr(), K_IN, 1, _stream()),
               "normalize inputs")
        Tn = torch.empty(n, N_OUT, device="cuda")
        out_rstd = torch.where(self.norm.out_std > 0, 1.0 / self.norm.out_std, torch.zeros_like(self.norm.out_std))
        _check(lib.rrtmg_sur_normalize(T.data_ptr(), T.stride(0), n, N_TARGETS, self.norm.out_mean.data_ptr(),
                                       out_rstd.data_ptr(), Tn.data_ptr(), N_OUT, 0, _stream()), "normalize targets")
        return X, Tn

    # -- forward / backward --------------------------------------------------
    def _buffers(self, B: int):
        import torch
        if getattr(self, "_buf_batch", None) == B:
            return self._buf
        bf, f32 = torch.bfloat16, torch.float32
        e = lambda *s, dt=f32: torch.empty(*s, device="cuda", dtype=dt)
        buf = dict(
            Xb=e(B, K_IN, dt=bf), Xbt=e(K_IN, B, dt=bf), Tb=e(B, N_OUT),
            Z=[e(B, HIDDEN) for _ in range(3)], H=[e(B, HIDDEN, dt=bf) for _ in range(3)],
            Ht=[e(HIDDEN, B, dt=bf) for _ in range(3)], Y=e(B, N_OUT),
            dY=e(B, N_OUT, dt=bf), dYt=e(N_OUT, B, dt=bf),
            dZ=[e(B, HIDDEN, dt=bf) for _ in range(3)], dZt=[e(HIDDEN, B, dt=bf) for _ in range(3)],
            gw=[torch.empty_like(w) for w in self.w], gb=[torch.empty_like(b) for b in self.b],
            loss=e(1),
        )
        self._ksplit = max(1, min(16, B // 1024))
        while B % (64 * self._ksplit):
            self._ksplit //= 2
        buf["part"] = e(self._ksplit * HIDDEN * max(K_IN, HIDDEN))
        self._buf, self._buf_batch = buf, B
        return buf

    def forward(self, X, *, Z=None, H=None, Ht=None, Y=None):
        """Y = MLP(X) for BF16 X [M, K_IN] (M a multiple of 128)."""
        import torch
        M = X.shape[0]
        inp = X
        for i in range(3):
            gemm_bf16(inp, self.wb[i], epilogue=_capi.EPI_GELU, bias=self.b[i], Z=None if Z is None else Z[i],
                      H=H[i], Ht=None if Ht is None else Ht[i])
            inp = H[i]
        if Y is None:
            Y = torch.empty(M, N_OUT, device="cuda")
        gemm_bf16(inp, self.wb[3], epilogue=_capi.EPI_F32, bias=self.b[3], C=Y)
        return Y

    def weight_image(self):
        """The BF16 weights packed for the fused inference kernel
        (rrtmg_sur_pack_weights), rebuilt after the weights change."""
        import torch
        img = getattr(self, "_wimg", None)
        if img is None or self._wimg_step != self.step:
            lib = _capi.load()
            img = torch.empty(_capi.WEIGHT_IMAGE_BYTES, device="cuda", dtype=torch.uint8)
            ptrs = (ctypes.c_void_p * 4)(*[w.data_ptr() for w in self.wb])
            _check(lib.rrtmg_sur_pack_weights(ctypes.byref(ptrs), img.data_ptr(), _stream()), "pack weights")
            self._wimg, self._wimg_step = img, self.step
        return img

    def train_step(self, X, Tn, idx, weights, *, lr: float, beta1=0.9, beta2=0.999, eps=1e-8,
                   weight_decay: float = 0.0) -> None:
        """One Adam step on the batch idx of (X, Tn); the batch loss is added to
        self._buf['loss'] (sum of weighted squared errors)."""
        lib = _capi.load()
        B = idx.shape[0]
        b = self._buffers(B)
        s = _stream()
        _check(lib.rrtmg_sur_gather(X.data_ptr(), K_IN, Tn.data_ptr(), N_OUT, idx.data_ptr(), B, b["Xb"].data_ptr(),
                                    b["Xbt"].data_ptr(), B, b["Tb"].data_ptr(), s), "gather")
        self.forward(b["Xb"], Z=b["Z"], H=b["H"], Ht=b["Ht"], Y=b["Y"])
        _check(lib.rrtmg_sur_loss_grad(b["Y"].data_ptr(), b["Tb"].data_ptr(), weights.data_ptr(), B, N_OUT,
                                       1.0 / (B * N_TARGETS), b["dY"].data_ptr(), b["dYt"].data_ptr(), B,
                                       b["loss"].data_ptr(), s), "loss gradient")
        ks = self._ksplit
        # layer 4 (linear), then the three GELU layers, last to first
        grads_in = (b["dYt"], b["dZt"][2], b["dZt"][1], b["dZt"][0])   # d(pre-activation)^T per layer 3..0
        acts_t = (b["Ht"][2], b["Ht"][1], b["Ht"][0], b["Xbt"])          # layer inputs^T
        for layer, gt, at in zip((3, 2, 1, 0), grads_in, acts_t):
            out_f, in_f = LAYER_SHAPES[layer]
            part = b["part"][:ks * out_f * in_f].view(ks, out_f, in_f)
            gemm_bf16(gt, at, epilogue=_capi.EPI_F32, C=part, ksplit=ks)
            _check(lib.rrtmg_sur_reduce_splits(part.data_ptr(), ks, out_f * in_f, b["gw"][layer].data_ptr(), s),
                   "reduce splits")
            _check(lib.rrtmg_sur_row_sum(gt.data_ptr(), B, out_f, B, b["gb"][layer].data_ptr(), s), "bias gradient")
            if layer > 0:
                g_rows = b["dY"] if layer == 3 else b["dZ"][layer]
                gemm_bf16(g_rows, self.wbt[layer], epilogue=_capi.EPI_DGELU, aux=b["Z"][layer - 1],
                          H=b["dZ"][layer - 1], Ht=b["dZt"][layer - 1])
        self.step += 1
        bc1, bc2 = 1.0 - beta1 ** self.step, 1.0 - beta2 ** self.step
        for i, (out_f, in_f) in enumerate(LAYER_SHAPES):
            a = _capi.SurAdamArgs(rows=out_f, cols=in_f, w=self.w[i].data_ptr(), m=self.mw[i].data_ptr(),
                                  v=self.vw[i].data_ptr(), grad=b["gw"][i].data_ptr(), lr=lr, beta1=beta1,
                                  beta2=beta2, eps=eps, bc1=bc1, bc2=bc2, weight_decay=weight_decay,
                                  wb=self.wb[i].data_ptr(), ldwb=in_f, wbt=self.wbt[i].data_ptr(), ldwbt=out_f)
            _check(lib.rrtmg_sur_adam(ctypes.byref(a), s), "adam (weights)")
            a = _capi.SurAdamArgs(rows=1, cols=out_f, w=self.b[i].data_ptr(), m=self.mb[i].data_ptr(),
                                  v=self.vb[i].data_ptr(), grad=b["gb"][i].data_ptr(), lr=lr, beta1=beta1,
                                  beta2=beta2, eps=eps, bc1=bc1, bc2=bc2, weight_decay=0.0)
            _check(lib.rrtmg_sur_adam(ctypes.byref(a), s), "adam (biases)")

    # -- persistence ----------------------------------------------------------
    def state(self) -> dict:
        out = {f"w{i}": w.cpu().numpy() for i, w in enumerate(self.w)}
        out.update({f"b{i}": b.cpu().numpy() for i, b in enumerate(self.b)})
        for k in ("in_mean", "in_rstd", "in_lo", "in_hi", "out_mean", "out_std"):
            out[k] = getattr(self.norm, k).cpu().numpy()
        out["step"] = np.array(self.step)
        return out

    def save(self, path) -> None:
        np.savez_compressed(path, **self.state())

    @classmethod
    def load(cls, path) -> "SurrogateModel":
        import torch
        z = np.load(path)
        m = cls.__new__(cls)
        m.w = [torch.from_numpy(z[f"w{i}"]).cuda() for i in range(len(LAYER_SHAPES))]
        m.b = [torch.from_numpy(z[f"b{i}"]).cuda() for i in range(len(LAYER_SHAPES))]
        m.wb = [w.to(torch.bfloat16).contiguous() for w in m.w]
        m.wbt = [w.t().contiguous().to(torch.bfloat16) for w in m.w]
        m.mw = [torch.zeros_like(w) for w in m.w]
        m.vw = [torch.zeros_like(w) for w in m.w]
        m.mb = [torch.zeros_like(b) for b in m.b]
        m.vb = [torch.zeros_like(b) for b in m.b]
        m.step = int(z["step"])
        m.norm = Normalization(*(torch.from_numpy(z[k]).cuda() for k in
                                 ("in_mean", "in_rstd", "in_lo", "in_hi", "out_mean", "out_std")))
        return m


def target_weights():
    """Loss weight per output: 1 for the 106 targets, 0 for the padding."""
    import torch
    w = torch.zeros(N_OUT, device="cuda")
    w[:N_TARGETS] = 1.0
    return w


def train(model: SurrogateModel, X, Tn, *, epochs: int, batch: int = 16384, lr: float = 1e-3, seed: int = 0,
          log=print) -> list[float]:
    """Adam with cosine learning-rate decay over `epochs` passes of (X, Tn);
    returns the mean normalized squared error of each epoch."""
    import torch
    n = X.shape[0]
    steps_per_epoch = n // batch
    total = epochs * steps_per_epoch
    w = target_weights()
    g = torch.Generator(device="cuda").manual_seed(seed)
    history = []
    step = 0
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g).to(torch.int32)
        model._buffers(batch)["loss"].zero_()
        for q in range(steps_per_epoch):
            rate = lr * 0.5 * (1.0 + math.cos(math.pi * step / max(1, total)))
            model.train_step(X, Tn, perm[q * batch:(q + 1) * batch], w, lr=rate)
            step += 1
        loss = float(model._buf["loss"].item()) / (steps_per_epoch * batch * N_TARGETS)
        history.append(loss)
        if log:
            log(f"epoch {ep + 1}/{epochs}: normalized MSE {loss:.5f}")
    return history


# ---------------------------------------------------------------------------
# inference with gate and plain-kernel fallback
# ---------------------------------------------------------------------------
@dataclass
class SurrogateResult:
    rthratenlw: object
    rthratensw: object
    glw: object
    lwupb: object
    swdnb: object
    swupb: object
    flags: object          # per column: 0 surrogate, 1 input range, 2 energy gate (bits)
    n_fallback: int


def infer(model: SurrogateModel, st, d: dict | None = None, *, energy_tol: float = 5.0,
          fallback: bool = True, fused: bool = True) -> SurrogateResult:
    """Surrogate radiation for a domain (synthetic.ColumnState; device fields d
    as torch CUDA tensors, built from st when None) with per-column gate and
    plain-kernel fallback.  fused: one kernel for the four layers and the
    decode (rrtmg_sur_mlp); otherwise one GEMM per layer and a decode kernel.
    Both give the same bits."""
    import torch
    lib = _capi.load()
    if st.nk != NK:
        raise ValueError(f"the surrogate is built for {NK} levels, got {st.nk}")
    d = d if d is not None else _device_fields(st, "cuda")
    nx, ny, nk = st.nx, st.ny, st.nk
    ncol = nx * ny
    mpad = (ncol + 127) // 128 * 128
    s = _stream()
    ws = _workspace(mpad, fused)
    flags = torch.empty(ncol, device="cuda", dtype=torch.int32)
    fa = _feature_args(d, nk, ny, ncol)
    fa.mean, fa.rstd = model.norm.in_mean.data_ptr(), model.norm.in_rstd.data_ptr()
    fa.X, fa.ldx, fa.x_layout = ws["X"].data_ptr(), K_IN, 1 if fused else 0
    fa.lo, fa.hi, fa.flags = model.norm.in_lo.data_ptr(), model.norm.in_hi.data_ptr(), flags.data_ptr()
    _check(lib.rrtmg_sur_features(ctypes.byref(fa), s), "features")
    out = dict(rthratenlw=torch.empty(nx, nk, ny, device="cuda"), rthratensw=torch.empty(nx, nk, ny, device="cuda"))
    for k in ("glw", "lwupb", "swdnb", "swupb"):
        out[k] = torch.empty(nx, ny, device="cuda")
    common = dict(ncol=ncol, nk=nk, ny=ny, out_mean=model.norm.out_mean.data_ptr(),
                  out_std=model.norm.out_std.data_ptr(), coszr=d["coszr"].data_ptr(), pi3d=d["pi3d"].data_ptr(),
                  p8w=d["p8w"].data_ptr(), energy_tol=energy_tol, flags=flags.data_ptr(),
                  **{k: v.data_ptr() for k, v in out.items()})
    if fused:
        ma = _capi.SurMlpArgs(X=ws["X"].data_ptr(), W=model.weight_image().data_ptr(), **common)
        for i in range(4):
            ma.bias[i] = model.b[i].data_ptr()
        _check(lib.rrtmg_sur_mlp(ctypes.byref(ma), s), "fused inference")
    else:
        Y = model.forward(ws["X"], H=ws["H"], Y=ws["Y"])
        da = _capi.SurDecodeArgs(Y=Y.data_ptr(), ldy=N_OUT, **common)
        _check(lib.rrtmg_sur_decode(ctypes.byref(da), s), "decode")
    n_fb = 0
    if fallback:
        n_fb = _fallback(st, d, flags, out)
    return SurrogateResult(flags=flags, n_fallback=n_fb, **out)


# Fields the network reads for every column (features and decode); the
# plain-kernel fallback also reads the other inputs, for its columns only.
NETWORK_FIELDS = ("t3d", "p3d", "qv3d", "qc3d", "qi3d", "qs3d", "cldfra3d", "o33d", "p8w", "pi3d", "tsk", "albedo",
                  "coszr", "emiss")
OUTPUT_FIELDS = ("rthratenlw", "rthratensw", "glw", "lwupb", "swdnb", "swupb")


def _network(model: SurrogateModel, d: dict, nx: int, ny: int, nk: int, out: dict, flags, energy_tol: float, X,
             s) -> None:
    """Features (tile layout) and the fused network with its decode and
    energy gate for an (nx, nk, ny) domain: device fields d, device outputs
    out, per-column flags; X holds at least ceil(nx ny / 128) feature tiles."""
    lib = _capi.load()
    ncol = nx * ny
    fa = _feature_args(d, nk, ny, ncol)
    fa.mean, fa.rstd = model.norm.in_mean.data_ptr(), model.norm.in_rstd.data_ptr()
    fa.X, fa.ldx, fa.x_layout = X.data_ptr(), K_IN, 1
    fa.lo, fa.hi, fa.flags = model.norm.in_lo.data_ptr(), model.norm.in_hi.data_ptr(), flags.data_ptr()
    _check(lib.rrtmg_sur_features(ctypes.byref(fa), s), "features")
    ma = _capi.SurMlpArgs(ncol=ncol, nk=nk, ny=ny, X=X.data_ptr(), W=model.weight_image().data_ptr(),
                          out_mean=model.norm.out_mean.data_ptr(), out_std=model.norm.out_std.data_ptr(),
                          coszr=d["coszr"].data_ptr(), pi3d=d["pi3d"].data_ptr(), p8w=d["p8w"].data_ptr(),
                          energy_tol=energy_tol, flags=flags.data_ptr(),
                          **{k: out[k].data_ptr() for k in OUTPUT_FIELDS})
    for i in range(4):
        ma.bias[i] = model.b[i].data_ptr()
    _check(lib.rrtmg_sur_mlp(ctypes.byref(ma), s), "fused inference")


_HOST_WS: dict = {}


def _host_workspace(nx: int, nk: int, ny: int, rows: int) -> dict:
    import torch
    key = (torch.cuda.current_device(), nx, nk, ny, rows)
    ws = _HOST_WS.get(key)
    if ws is None:
        dev = "cuda"
        shapes = {k: (nx, nk + 1, ny) if k == "p8w" else ((nx, ny) if k in ("tsk", "albedo", "coszr", "emiss")
                                                          else (nx, nk, ny)) for k in NETWORK_FIELDS}
        ws = dict(d={k: torch.empty(v, device=dev) for k, v in shapes.items()},
                  out={k: torch.empty((nx, nk, ny) if k.startswith("rthraten") else (nx, ny), device=dev)
                       for k in OUTPUT_FIELDS},
                  flags=torch.empty(nx * ny, device=dev, dtype=torch.int32),
                  X=torch.zeros((rows * ny + 127) // 128 * 128, K_IN, device=dev, dtype=torch.bfloat16),
                  h2d=torch.cuda.Stream(), d2h=torch.cuda.Stream())
        _HOST_WS.clear()  # keep one domain shape resident
        _HOST_WS[key] = ws
    return ws


def _slab_bounds(nx: int, slabs: int) -> list:
    """West-east row ranges of the host pipeline's slabs: equal slabs, the
    last two at a half and a quarter of the others; no empty slab."""
    slabs = max(1, min(int(slabs), nx))
    weights = [1.0] * slabs if slabs < 3 else [1.0] * (slabs - 2) + [0.5, 0.25]
    total, acc, edges = sum(weights), 0.0, [0]
    for w in weights[:-1]:
        acc += w
        edges.append(int(round(nx * acc / total)))
    edges.append(nx)
    return [(i0, i1) for i0, i1 in zip(edges, edges[1:]) if i1 > i0]


def infer_host(model: SurrogateModel, st, host: dict, out: dict, *, energy_tol: float = 5.0, slabs: int = 8,
               fallback: bool = True) -> int:
    """Surrogate radiation with host inputs and outputs, pipelined over the
    host link: `host` holds every input field of the domain as page-locked
    CPU float32 tensors (st's shapes), `out` the six output fields
    (rthratenlw, rthratensw, glw, lwupb, swdnb, swupb) as page-locked CPU
    float32 tensors.  The network's fields go to the GPU in `slabs` slabs of
    west-east rows on one copy stream, each slab's network runs as soon as it
    has landed and its outputs return on a second copy stream; the fallback
    then reads the other inputs of its columns from host memory in place and
    writes its columns' outputs back to host memory in place.  The last two
    slabs are a half and a quarter of the others, which shortens the part of
    the step left after the last transfer (the last slab's network and the
    return of its outputs).  Results are those of infer() on device fields.
    Returns the number of fallback columns; the outputs are complete on
    return."""
    import torch
    if st.nk != NK:
        raise ValueError(f"the surrogate is built for {NK} levels, got {st.nk}")
    for name, t in list(host.items()) + list(out.items()):
        if not (isinstance(t, torch.Tensor) and not t.is_cuda and t.is_pinned() and t.is_contiguous()
                and t.dtype == torch.float32):
            raise ValueError(f"{name} must be a contiguous page-locked CPU float32 tensor")
    nx, ny, nk = st.nx, st.ny, st.nk
    bounds = _slab_bounds(nx, slabs)
    ws = _host_workspace(nx, nk, ny, max(i1 - i0 for i0, i1 in bounds))
    main, h2d, d2h = torch.cuda.current_stream(), ws["h2d"], ws["d2h"]
    dev, dout, flags = ws["d"], ws["out"], ws["flags"]
    h2d.wait_stream(main)  # earlier work on these buffers is done
    d2h.wait_stream(main)
    landed = []
    with torch.cuda.stream(h2d):
        for i0, i1 in bounds:
            for k in NETWORK_FIELDS:
                dev[k][i0:i1].copy_(host[k][i0:i1], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(h2d)
            landed.append(ev)
    s = _stream()
    n_fb = 0
    for (i0, i1), ev in zip(bounds, landed):
        main.wait_event(ev)
        d_slab = {k: v[i0:i1] for k, v in dev.items()}
        o_slab = {k: v[i0:i1] for k, v in dout.items()}
        _network(model, d_slab, i1 - i0, ny, nk, o_slab, flags[i0 * ny:i1 * ny], energy_tol, ws["X"], s)
        done = torch.cuda.Event()
        done.record(main)
        d2h.wait_event(done)
        with torch.cuda.stream(d2h):
            for k in OUTPUT_FIELDS:
                out[k][i0:i1].copy_(dout[k][i0:i1], non_blocking=True)
    if fallback:
        # the fallback reads its columns' other inputs from host memory in
        # place; a slab's fallback ahead of the later slabs' transfers gained
        # nothing (the last one is latency-bound and stays exposed)
        returned = torch.cuda.Event()
        returned.record(d2h)
        src = {k: (dev[k] if k in dev else host[k]) for k in host}
        n_fb = _fallback(st, src, flags, out, before_scatter=returned)
    main.wait_stream(d2h)
    main.synchronize()
    return n_fb


def fused_kernel_call(model: SurrogateModel, st, d: dict, *, energy_tol: float = 5.0):
    """Runs the features of a 50-level domain once and returns a callable that
    launches only the fused inference kernel on them (for timing and
    profiling the dominant kernel); outputs land in fresh device buffers."""
    import torch
    lib = _capi.load()
    nx, ny, nk = st.nx, st.ny, st.nk
    ncol = nx * ny
    mpad = (ncol + 127) // 128 * 128
    s = _stream()
    X = torch.zeros(mpad, K_IN, device="cuda", dtype=torch.bfloat16)
    flags = torch.empty(ncol, device="cuda", dtype=torch.int32)
    fa = _feature_args(d, nk, ny, ncol)
    fa.mean, fa.rstd = model.norm.in_mean.data_ptr(), model.norm.in_rstd.data_ptr()
    fa.X, fa.ldx, fa.x_layout = X.data_ptr(), K_IN, 1
    fa.lo, fa.hi, fa.flags = model.norm.in_lo.data_ptr(), model.norm.in_hi.data_ptr(), flags.data_ptr()
    _check(lib.rrtmg_sur_features(ctypes.byref(fa), s), "features")
    out = dict(rthratenlw=torch.empty(nx, nk, ny, device="cuda"), rthratensw=torch.empty(nx, nk, ny, device="cuda"))
    for k in ("glw", "lwupb", "swdnb", "swupb"):
        out[k] = torch.empty(nx, ny, device="cuda")
    ma = _capi.SurMlpArgs(ncol=ncol, nk=nk, ny=ny, X=X.data_ptr(), W=model.weight_image().data_ptr(),
                          out_mean=model.norm.out_mean.data_ptr(), out_std=model.norm.out_std.data_ptr(),
                          coszr=d["coszr"].data_ptr(), pi3d=d["pi3d"].data_ptr(), p8w=d["p8w"].data_ptr(),
                          energy_tol=energy_tol, flags=flags.data_ptr(), **{k: v.data_ptr() for k, v in out.items()})
    for i in range(4):
        ma.bias[i] = model.b[i].data_ptr()
    keep = (X, flags, out, ma)

    def call():
        _check(lib.rrtmg_sur_mlp(ctypes.byref(keep[3]), _stream()), "fused inference")
    call.buffers = keep
    return call


_WORKSPACES: dict = {}


def _workspace(mpad: int, fused: bool) -> dict:
    """Network buffers for mpad rows, kept per device and reused by every call
    with the same padded column count and path (the calls on one device are
    ordered on its stream).  X starts zero; the fused path needs only X (in
    the 128-row tile layout), the unfused one also the hidden activations and
    the outputs."""
    import torch
    key = (torch.cuda.current_device(), mpad, fused)
    ws = _WORKSPACES.get(key)
    if ws is None:
        bf = torch.bfloat16
        ws = dict(X=torch.zeros(mpad, K_IN, device="cuda", dtype=bf))
        if not fused:
            ws["H"] = [torch.empty(mpad, HIDDEN, device="cuda", dtype=bf) for _ in range(3)]
            ws["Y"] = torch.empty(mpad, N_OUT, device="cuda")
        _WORKSPACES.clear()  # keep one domain size resident
        _WORKSPACES[key] = ws
    return ws


_FIELDS_3D = ("p3d", "pi3d", "t3d", "dz8w", "qv3d", "qc3d", "qi3d", "qs3d", "cldfra3d", "o33d", "re_cloud",
              "re_ice", "re_snow")
_FIELDS_LEV = ("p8w", "t8w")
_FIELDS_2D = ("tsk", "emiss", "albedo", "coszr", "xland", "xice", "snow")


_SIDE = {}
_HIGH = {}


def _side_stream():
    import torch
    dev = torch.cuda.current_device()
    if dev not in _SIDE:
        _SIDE[dev] = torch.cuda.Stream(device=dev)
    return _SIDE[dev]


def _high_stream():
    """A stream of the device's highest priority: its blocks are dispatched
    before those of default-priority streams as SMs free up."""
    import torch
    dev = torch.cuda.current_device()
    if dev not in _HIGH:
        _HIGH[dev] = torch.cuda.Stream(device=dev, priority=-100)  # clamped to the highest
    return _HIGH[dev]


_SCALAR_KEYS_LW = ("p_top", "yr", "co2vmr", "n2ovmr", "ch4vmr", "cfc11vmr", "cfc12vmr", "has_reqc", "has_reqi",
                   "has_reqs", "icloud", "cldovrlp")
_SCALAR_KEYS_SW = ("solcon", "yr", "co2vmr", "n2ovmr", "ch4vmr", "has_reqc", "has_reqi", "has_reqs", "icloud",
                   "cldovrlp")


class _FallbackPlan:
    """Persistent buffers and prebuilt C-ABI arguments of the plain-kernel
    fallback for up to `cap` columns of nk levels: the gathered input fields
    and the LW/SW outputs of a compact (1, nk, n) domain (n <= cap, each
    field's first n columns per level), so a call allocates nothing and
    issues one gather, the LW and SW calls and one scatter."""

    def __init__(self, nk: int, cap: int, lw_scalars: dict, sw_scalars: dict):
        import torch
        from . import rrtmg
        self.nk, self.cap = nk, cap
        self.ctx = rrtmg.default_context()
        dev = "cuda"
        nz = {k: nk for k in _FIELDS_3D}
        nz.update({k: nk + 1 for k in _FIELDS_LEV})
        nz.update({k: 1 for k in _FIELDS_2D})
        self.nz = nz
        self.sub = {k: torch.empty(z * cap, device=dev) for k, z in nz.items()}
        self.lw_out = {k: torch.empty((nk if k.startswith("rthraten") else 1) * cap, device=dev)
                       for k in _capi.LW_OUT_FIELDS}
        self.sw_out = {k: torch.empty((nk if k.startswith("rthraten") else 1) * cap, device=dev)
                       for k in _capi.SW_OUT_FIELDS}
        self.cfg_lw = rrtmg.lw_config(1, 1, nk, **lw_scalars)
        self.cfg_sw = rrtmg.sw_config(1, 1, nk, **sw_scalars)
        self.cin_lw = _capi.LwIn(**{k: self.sub[k].data_ptr() for k in _capi.LW_IN_FIELDS})
        self.cout_lw = _capi.LwOut(**{k: v.data_ptr() for k, v in self.lw_out.items()})
        self.cin_sw = _capi.SwIn(**{k: self.sub[k].data_ptr() for k in _capi.SW_IN_FIELDS})
        self.cout_sw = _capi.SwOut(**{k: v.data_ptr() for k, v in self.sw_out.items()})
        self.gather = _capi.SurFields(nfields=len(nz))
        for i, (k, z) in enumerate(nz.items()):
            self.gather.dst[i] = self.sub[k].data_ptr()
            self.gather.nz[i] = z
        self.scatter_src = (("rthratenlw", self.lw_out["rthratenlw"], nk), ("rthratensw", self.sw_out["rthratensw"], nk),
                            ("glw", self.lw_out["glw"], 1), ("lwupb", self.lw_out["lwupb"], 1),
                            ("swdnb", self.sw_out["swdnb"], 1), ("swupb", self.sw_out["swupb"], 1))
        self.scatter = _capi.SurFields(nfields=len(self.scatter_src))
        for i, (_, t, z) in enumerate(self.scatter_src):
            self.scatter.src[i] = t.data_ptr()
            self.scatter.nz[i] = z


_PLANS: dict = {}
_LISTS: dict = {}


def _fallback_plan(st, n: int) -> _FallbackPlan:
    import torch
    cap = 256
    while cap < n:
        cap *= 2
    lw_kw, sw_kw = st.lw_kwargs(), st.sw_kwargs()
    lw_s = {k: lw_kw[k] for k in _SCALAR_KEYS_LW if k in lw_kw}
    sw_s = {k: sw_kw[k] for k in _SCALAR_KEYS_SW if k in sw_kw}
    key = (torch.cuda.current_device(), st.nk, cap, tuple(sorted(lw_s.items())), tuple(sorted(sw_s.items())))
    plan = _PLANS.get(key)
    if plan is None:
        plan = _FallbackPlan(st.nk, cap, lw_s, sw_s)
        while len(_PLANS) >= 2:  # keep the capacity plan and one exact-size plan resident
            _PLANS.pop(next(iter(_PLANS)))
        _PLANS[key] = plan
    return plan


# Columns the fallback re-solves without reading their number on the host;
# when the gate rejects more, those steps take the synchronous path as well.
FALLBACK_CAPACITY = 2048


def _fallback(st, d: dict, flags, out: dict, before_scatter=None) -> int:
    """Re-solve the flagged columns with the plain kernels, writing their
    surrogate outputs over; returns how many columns were re-solved.  The
    gather, the LW and SW calls and the scatter are queued with the column
    count left on the device (rrtmg_lwrad_live / rrtmg_swrad_live over a
    compact domain of a fixed capacity); the count is read once at the end.
    Steps with more rejected columns than the capacity re-solve all of them
    again on a domain of the exact size.  d and out may hold page-locked host
    tensors, which the gathers read and the scatters write in place;
    before_scatter: an event the scatters wait for."""
    import torch
    lib = _capi.load()
    s = _stream()
    nx, ny, nk = st.nx, st.ny, st.nk
    ncol = nx * ny
    key = (torch.cuda.current_device(), ncol)
    if key not in _LISTS:
        _LISTS.clear()
        _LISTS[key] = (torch.empty(ncol, device="cuda", dtype=torch.int32),
                       torch.zeros(1, device="cuda", dtype=torch.int32))
    lst, cnt = _LISTS[key]
    cnt.zero_()
    _check(lib.rrtmg_sur_compact(flags.data_ptr(), ncol, lst.data_ptr(), cnt.data_ptr(), s), "compact")
    plan = _fallback_plan(st, min(ncol, FALLBACK_CAPACITY))
    _solve_listed(plan, lib, s, lst, cnt, ny, d, out, before_scatter, live=True)
    n = int(cnt.item())
    if n > plan.cap:
        _solve_listed(_fallback_plan(st, n), lib, s, lst, cnt, ny, d, out, before_scatter, live=False, n=n)
    return n


def _solve_listed(plan, lib, s, lst, cnt, ny, d, out, before_scatter, *, live: bool, n: int | None = None) -> None:
    """Gather the listed columns into the plan's compact domain, run LW (side
    stream) and SW (high-priority stream) on it, scatter the results back.
    live: the domain has plan.cap slots and the count stays on the device;
    else exactly n columns."""
    import torch
    m = plan.cap if live else n
    for i, k in enumerate(plan.nz):
        plan.gather.src[i] = d[k].data_ptr()
    _check(lib.rrtmg_sur_move_fields(lst.data_ptr(), cnt.data_ptr(), m, ny, ctypes.byref(plan.gather), 1, m, 0, s),
           "gather")
    plan.cfg_lw.ny = m
    plan.cfg_sw.ny = m
    ctx = plan.ctx
    # LW and SW on two streams forked from the current one; both read the
    # gathered fields, and the current stream waits for both before the
    # scatter.  SW, the longer chain at fallback sizes (its latency-bound
    # sweep follows throughput-bound optics), runs at high priority so that
    # LW's blocks fill the SMs its kernels leave free rather than delay it.
    main, side, high = torch.cuda.current_stream(), _side_stream(), _high_stream()
    ready = torch.cuda.Event()
    ready.record(main)
    side.wait_event(ready)
    high.wait_event(ready)
    side_s, high_s = ctypes.c_void_p(side.cuda_stream), ctypes.c_void_p(high.cuda_stream)
    if live:
        ctx.check(ctx.lib.rrtmg_lwrad_live(ctx.handle, ctypes.byref(plan.cfg_lw), ctypes.byref(plan.cin_lw),
                                           ctypes.byref(plan.cout_lw), ctypes.c_void_p(cnt.data_ptr()), side_s))
        ctx.check(ctx.lib.rrtmg_swrad_live(ctx.handle, ctypes.byref(plan.cfg_sw), ctypes.byref(plan.cin_sw),
                                           ctypes.byref(plan.cout_sw), ctypes.c_void_p(cnt.data_ptr()), high_s))
    else:
        ctx.check(ctx.lib.rrtmg_lwrad(ctx.handle, ctypes.byref(plan.cfg_lw), ctypes.byref(plan.cin_lw),
                                      ctypes.byref(plan.cout_lw), side_s))
        ctx.check(ctx.lib.rrtmg_swrad(ctx.handle, ctypes.byref(plan.cfg_sw), ctypes.byref(plan.cin_sw),
                                      ctypes.byref(plan.cout_sw), high_s))
    for done_on in (side, high):
        done = torch.cuda.Event()
        done.record(done_on)
        main.wait_event(done)
    if before_scatter is not None:
        main.wait_event(before_scatter)
    for i, (k, _, _) in enumerate(plan.scatter_src):
        plan.scatter.dst[i] = out[k].data_ptr()
    _check(lib.rrtmg_sur_move_fields(lst.data_ptr(), cnt.data_ptr(), m, ny, ctypes.byref(plan.scatter), 0, m, 0, s),
           "scatter")


def heating_kday(rthraten, pi3d):
    """Heating rate in K/day from a theta tendency (rthraten * 86400 * pi3d)."""
    return rthraten * 86400.0 * pi3d
