"""The tcgen05 GEMM's bounded waits, made to run out on purpose and in the
allowed form: a wait on an mbarrier phase that nothing completes.

With rrtmg_gemm_test_withhold_commit on, each CTA withholds the tensor-core
commit of its first K block, so its wait for that block (limit set to 20 us
through rrtmg_gemm_set_wait_ns) gives up.  The CTA then waits for its second
block's commit, which covers every MMA it issued, frees its tensor memory and
writes nothing; rrtmg_gemm_error returns RRTMG_TIMEOUT.  Nothing is left in
flight: the GEMM stages its operands with cp.async, which the CTA waits for
before it leaves.  A normal call on the same process afterwards must give the
bits of a call made before the timeout.
"""

from __future__ import annotations

import ctypes

import pytest

pytestmark = pytest.mark.gpu

RRTMG_OK, RRTMG_BAD_ARG, RRTMG_TIMEOUT = 0, 1, 4


@pytest.fixture()
def gemm_env(pkg):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wrf_jax_b200 import _capi, surrogate
    lib = _capi.load()
    assert lib.rrtmg_gemm_set_tile(0) == RRTMG_OK
    yield torch, lib, surrogate, _capi
    lib.rrtmg_gemm_test_withhold_commit(0)
    lib.rrtmg_gemm_set_wait_ns(0)
    torch.cuda.synchronize()
    surrogate.gemm_error(reset=True)


def _args(_capi, A, B, C, M, N, K):
    a = _capi.GemmArgs()
    a.A, a.lda, a.B, a.ldb = A.data_ptr(), K, B.data_ptr(), K
    a.M, a.N, a.K, a.ksplit, a.epilogue = M, N, K, 1, _capi.EPI_F32
    a.bias, a.C, a.ldc, a.split_stride = None, C.data_ptr(), N, 0
    return a


def test_withheld_commit_times_out_then_next_call_is_exact(gemm_env):
    torch, lib, surrogate, _capi = gemm_env
    M, N, K = 256, 256, 256  # 4 K blocks > 3 pipeline stages of the 256-wide tile
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = (torch.randn(N, K, device="cuda", generator=g) / K ** 0.5).bfloat16()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    surrogate.gemm_error(reset=True)

    ref = torch.full((M, N), float("nan"), device="cuda")
    assert lib.rrtmg_gemm_bf16(ctypes.byref(_args(_capi, A, B, ref, M, N, K)), stream) == RRTMG_OK
    torch.cuda.synchronize()
    flag = ctypes.c_uint(7)
    assert lib.rrtmg_gemm_error(1, ctypes.byref(flag)) == RRTMG_OK and flag.value == 0
    assert not torch.isnan(ref).any()

    # the timeout: a 20 us limit and the first block's commit withheld
    assert lib.rrtmg_gemm_set_wait_ns(20000) == RRTMG_OK
    assert lib.rrtmg_gemm_test_withhold_commit(1) == RRTMG_OK
    out = torch.full((M, N), float("nan"), device="cuda")
    assert lib.rrtmg_gemm_bf16(ctypes.byref(_args(_capi, A, B, out, M, N, K)), stream) == RRTMG_OK
    torch.cuda.synchronize()
    assert lib.rrtmg_gemm_error(1, ctypes.byref(flag)) == RRTMG_TIMEOUT
    assert flag.value != 0
    assert torch.isnan(out).all()  # a CTA that gave up writes no output
    # a call too short to drain behind the withheld commit is refused on the host
    short = torch.empty(M, N, device="cuda")
    assert lib.rrtmg_gemm_bf16(ctypes.byref(_args(_capi, A, B, short, M, N, 192)), stream) == RRTMG_BAD_ARG

    # back to normal: the same context computes the same bits
    assert lib.rrtmg_gemm_test_withhold_commit(0) == RRTMG_OK
    assert lib.rrtmg_gemm_set_wait_ns(0) == RRTMG_OK
    again = torch.full((M, N), float("nan"), device="cuda")
    assert lib.rrtmg_gemm_bf16(ctypes.byref(_args(_capi, A, B, again, M, N, K)), stream) == RRTMG_OK
    torch.cuda.synchronize()
    assert lib.rrtmg_gemm_error(1, ctypes.byref(flag)) == RRTMG_OK and flag.value == 0
    assert torch.equal(again.view(torch.int32), ref.view(torch.int32))
