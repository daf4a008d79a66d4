"""tcgen05 BF16 GEMM (sphg_gemm_bf16_tn) against an fp32 product of the same
bf16 inputs: C = A B^T, accumulate, split-K, every N tile width."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K,acc,split", [(128, 128, 64, 0, 1), (256, 128, 192, 0, 1), (384, 64, 256, 1, 1),
                                             (128, 16, 128, 0, 1), (256, 32, 64, 0, 1), (128, 384, 320, 0, 1),
                                             (512, 128, 1024, 1, 4), (128, 48, 64, 0, 1)])
def test_gemm_matches_fp32_reference(cuda_ok, lib, M, N, K, acc, split):
    import torch
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N * 3 + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C0 = torch.randn(M, N, device="cuda", generator=g)
    C = C0.clone() if (acc or split > 1) else torch.zeros(M, N, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.sphg_gemm_bf16_tn(A.data_ptr(), B.data_ptr(), C.data_ptr(), M, N, K, acc, split, err.data_ptr(),
                               torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == 0 and int(err.item()) == 0
    ref = A.float() @ B.float().T
    if acc or split > 1:
        ref = ref + C0
    scale = float(ref.abs().max())
    assert float((C - ref).abs().max()) <= 1e-4 * scale * (K / 64) ** 0.5, float((C - ref).abs().max()) / scale


def test_gemm_rejects_bad_shapes(lib):
    import ctypes
    one = ctypes.c_void_p(16)
    assert lib.sphg_gemm_bf16_tn(one, one, one, 100, 128, 64, 0, 1, one, None) != 0   # M % 128
    assert lib.sphg_gemm_bf16_tn(one, one, one, 128, 24, 64, 0, 1, one, None) != 0    # N % 16
    assert lib.sphg_gemm_bf16_tn(one, one, one, 128, 128, 32, 0, 1, one, None) != 0   # K % 64
