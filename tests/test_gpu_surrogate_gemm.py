"""The surrogate's hand-written tcgen05 BF16 GEMM (grrt_surrogate_gemm_bf16)
against a float64 product of the same BF16 operands.

Bar: FP32 accumulation of exact BF16 products differs from the float64 sum
only by accumulation rounding, so |C - C64| <= 1e-5 * sum_k |A_ik B_jk| + 1e-6
for every element; BF16 outputs are within one BF16 rounding (2^-8 relative)
of the float64 value after the epilogue.
"""
import pytest
import torch

pytestmark = pytest.mark.gpu


def gemm(grrt, A, B, splits=1, bias=None, gate=None, act=0, f32=True, bf16=False):
    M, K = A.shape
    N = B.shape[0]
    out32 = torch.full((splits, M, N), float("nan"), dtype=torch.float32, device="cuda") if f32 else None
    out16 = torch.full((M, N), float("nan"), dtype=torch.bfloat16, device="cuda") if bf16 else None
    L = grrt.lib()
    rc = L.grrt_surrogate_gemm_bf16(A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), M, N, K, splits,
                                    bias.data_ptr() if bias is not None else None,
                                    gate.data_ptr() if gate is not None else None, N, act,
                                    out32.data_ptr() if f32 else None, N,
                                    out16.data_ptr() if bf16 else None, N, None)
    assert rc == 0
    return out32, out16


def ref(A, B):
    a, b = A.double(), B.double()
    return a @ b.T, a.abs() @ b.abs().T


SHAPES = [(128, 16, 64), (100, 32, 64), (300, 256, 256), (1000, 64, 512), (4096, 256, 256), (257, 128, 1024)]


@pytest.mark.parametrize("M,N,K", SHAPES)
def test_gemm_matches_float64(grrt, need_gpu, M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    out, _ = gemm(grrt, A, B)
    c, mag = ref(A, B)
    err = (out[0].double() - c).abs()
    bound = 1e-5 * mag + 1e-6
    assert bool((err <= bound).all()), f"max err {float(err.max()):.3e}, worst ratio {float((err / bound).max()):.2f}"


def test_gemm_split_k_partials_sum(grrt, need_gpu):
    M, N, K = 256, 256, 64 * 40
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = torch.randn(N, K, device="cuda", generator=g).bfloat16()
    out, _ = gemm(grrt, A, B, splits=8)  # 40 K-blocks over 8 splits of 5
    c, mag = ref(A, B)
    err = (out.double().sum(0) - c).abs()
    assert bool((err <= 1e-5 * mag + 1e-6).all())


def test_gemm_epilogue_bias_silu_and_gate(grrt, need_gpu):
    M, N, K = 384, 256, 128
    g = torch.Generator(device="cuda").manual_seed(11)
    A = torch.randn(M, K, device="cuda", generator=g).bfloat16()
    B = (0.1 * torch.randn(N, K, device="cuda", generator=g)).bfloat16()
    bias = torch.randn(N, device="cuda", generator=g)
    z32, h16 = gemm(grrt, A, B, bias=bias, act=1, bf16=True)
    c, mag = ref(A, B)
    z = c + bias.double()
    assert bool(((z32[0].double() - z).abs() <= 1e-5 * mag + 1e-5).all())
    h = z * torch.sigmoid(z)
    assert bool(((h16.double() - h).abs() <= 2.0 ** -8 * h.abs() + 1e-4).all())
    gate = torch.randn(M, N, device="cuda", generator=g)
    d32, _ = gemm(grrt, A, B, gate=gate)
    s = torch.sigmoid(gate.double())
    want = c * s * (1 + gate.double() * (1 - s))
    assert bool(((d32[0].double() - want).abs() <= 1e-4 * (mag + 1)).all())


def test_gemm_rejects_bad_shapes(grrt):
    L = grrt.lib()
    # N not a multiple of 16, K not a multiple of 64: refused before any launch
    assert L.grrt_surrogate_gemm_bf16(1, 64, 1, 64, 128, 24, 64, 1, None, None, 0, 0, 1, 24, None, 0, None) == -1
    assert L.grrt_surrogate_gemm_bf16(1, 64, 1, 64, 128, 16, 48, 1, None, None, 0, 0, 1, 16, None, 0, None) == -1
