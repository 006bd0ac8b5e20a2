"""tcgen05 BF16 GEMM of the surrogate against a plain torch fp32 reference of
the same op (fp32 matmul of the bf16-rounded operands).  Tolerances: fp32
accumulation in a different order, |diff| <= 1e-4 * sqrt(K) * scale; bf16
outputs within one bf16 rounding (relative 2^-8) of the reference value."""

from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _operands(torch, M, N, K, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = (torch.randn(N, K, device="cuda", generator=g) / K ** 0.5).bfloat16()
    bias = torch.randn(N, device="cuda", generator=g) * 0.1
    return A, B, bias


@pytest.mark.parametrize("M,N,K,ksplit", [(128, 128, 64, 1), (256, 384, 512, 1), (512, 128, 1024, 4),
                                         (384, 512, 192, 1), (256, 256, 2048, 8)])
def test_gemm_f32_matches_torch(torch_cuda, M, N, K, ksplit):
    torch = torch_cuda
    from wrf_jax_b200 import surrogate, _capi
    A, B, bias = _operands(torch, M, N, K, 1)
    C = torch.empty(ksplit, M, N, device="cuda")
    surrogate.gemm_bf16(A, B, epilogue=_capi.EPI_F32, bias=bias, C=C, ksplit=ksplit)
    torch.cuda.synchronize()
    assert surrogate.gemm_error() == 0
    ref = A.float() @ B.float().T + bias
    got = C.sum(0)
    torch.testing.assert_close(got, ref, rtol=1e-4, atol=1e-4 * K ** 0.5)


def test_gemm_gelu_epilogue(torch_cuda):
    torch = torch_cuda
    from wrf_jax_b200 import surrogate, _capi
    M, N, K = 256, 256, 512
    A, B, bias = _operands(torch, M, N, K, 2)
    Z = torch.empty(M, N, device="cuda")
    H = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
    Ht = torch.empty(N, M, device="cuda", dtype=torch.bfloat16)
    surrogate.gemm_bf16(A, B, epilogue=_capi.EPI_GELU, bias=bias, Z=Z, H=H, Ht=Ht)
    torch.cuda.synchronize()
    assert surrogate.gemm_error() == 0
    zref = A.float() @ B.float().T + bias
    torch.testing.assert_close(Z, zref, rtol=1e-4, atol=1e-3)
    # GELU in the tanh form with the hardware tanh (relative error about
    # 2^-11) and a BF16 result: within one BF16 unit of the exact tanh form
    href = torch.nn.functional.gelu(Z, approximate="tanh")
    torch.testing.assert_close(H.float(), href, rtol=2 ** -7, atol=2e-3)
    torch.testing.assert_close(Ht.float().T, H.float(), rtol=0, atol=0)


def test_gemm_dgelu_epilogue(torch_cuda):
    torch = torch_cuda
    from wrf_jax_b200 import surrogate, _capi
    M, N, K = 128, 256, 256
    A, B, _ = _operands(torch, M, N, K, 3)
    aux = torch.randn(M, N, device="cuda")
    H = torch.empty(M, N, device="cuda", dtype=torch.bfloat16)
    Ht = torch.empty(N, M, device="cuda", dtype=torch.bfloat16)
    surrogate.gemm_bf16(A, B, epilogue=_capi.EPI_DGELU, aux=aux, H=H, Ht=Ht)
    torch.cuda.synchronize()
    z = aux.clone().requires_grad_(True)
    torch.nn.functional.gelu(z, approximate="tanh").sum().backward()
    acc = A.float() @ B.float().T
    ref = acc * z.grad
    # GELU' with the hardware tanh (relative error about 2^-11 in tanh, so
    # about 1e-3 absolute in GELU'), scaled by the accumulator, in BF16
    torch.testing.assert_close(H.float(), ref, rtol=2 ** -7, atol=2e-3 * float(acc.abs().max()))
    torch.testing.assert_close(Ht.float().T, H.float(), rtol=0, atol=0)


def test_gemm_rejects_unaligned_shapes(torch_cuda):
    torch = torch_cuda
    from wrf_jax_b200 import surrogate
    A = torch.zeros(100, 64, device="cuda", dtype=torch.bfloat16)
    B = torch.zeros(128, 64, device="cuda", dtype=torch.bfloat16)
    C = torch.zeros(100, 128, device="cuda")
    with pytest.raises(ValueError):
        surrogate.gemm_bf16(A, B, C=C)
