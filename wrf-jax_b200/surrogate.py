"""Learned radiation surrogate: an MLP from a column profile to LW/SW heating
profiles and surface fluxes, trained and run on B200 tensor cores.

Every arithmetic step of training and inference runs in librrtmg_b200.so:
tcgen05 BF16 GEMMs with fused bias/GELU epilogues (include/rrtmg_surrogate.h)
and small CUDA kernels for features, loss, bias gradients and Adam.  torch is
used only to hold device buffers and streams.
"""

from __future__ import annotations

import ctypes

from . import _capi


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def gemm_bf16(A, B, *, epilogue: int = _capi.EPI_F32, bias=None, C=None, ksplit: int = 1, H=None, Ht=None,
              aux=None, Z=None, stream=None) -> None:
    """C[M x N] = A[M x K] @ B[N x K]^T on the tensor cores, with the epilogue
    of include/rrtmg_surrogate.h.  A and B are contiguous bf16 CUDA tensors;
    outputs are preallocated tensors (C: float32 [ksplit, M, N] or [M, N];
    H: bf16 [M, N]; Ht: bf16 [N, M]; Z, aux: float32 [M, N])."""
    import torch

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
    s = stream if stream is not None else torch.cuda.current_stream().cuda_stream
    st = lib.rrtmg_gemm_bf16(ctypes.byref(g), ctypes.c_void_p(s))
    if st != 0:
        raise ValueError(f"rrtmg_gemm_bf16 rejected the arguments (status {st}): M={M} N={N} K={K} ksplit={ksplit}")


def gemm_error(reset: bool = True) -> int:
    """Synchronous read of the GEMM timeout flag (0 = no CTA gave up)."""
    flag = ctypes.c_uint(0)
    st = _capi.load().rrtmg_gemm_error(int(reset), ctypes.byref(flag))
    if st != 0:
        raise RuntimeError(f"rrtmg_gemm_error failed with status {st}")
    return flag.value
