"""tcgen05 BF16 GEMM of the surrogate MLP against a plain PyTorch FP32 matmul
of the same BF16 operands (FP32 accumulation on both sides)."""
import ctypes

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from pelelmex_b200 import _lib  # noqa: E402

DEV = "cuda:0"
EPI_F32, EPI_BF16, EPI_GELU, EPI_DGELU = 0, 1, 2, 3


def gelu(x):
    return 0.5 * x * (1.0 + torch.tanh(0.7978845608028654 * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    u = 0.7978845608028654 * (x + 0.044715 * x ** 3)
    t = torch.tanh(u)
    return 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * 0.7978845608028654 * (1 + 3 * 0.044715 * x * x)


def gemm(A, B, bias=None, epi=EPI_F32, aux=None, n_valid=0):
    M, K = A.shape
    N = B.shape[0]
    out = torch.empty((M, N), device=DEV, dtype=torch.float32 if epi == EPI_F32 else torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    L = _lib.load()
    code = L.b200chem_mlp_gemm_bf16(A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0), M, N, K, out.data_ptr(),
                                    out.stride(0), bias.data_ptr() if bias is not None else None,
                                    aux.data_ptr() if aux is not None else None, epi, n_valid, err.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream)
    assert code == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0, "mbarrier wait timed out"
    return out


@pytest.mark.parametrize("M,N,K", [(128, 16, 16), (128, 32, 32), (256, 256, 256), (384, 32, 256), (256, 256, 1024),
                                   (128, 512, 64), (1024, 256, 32),
                                   # many tiles per CTA: the two accumulators and the stage ring wrap around
                                   (128 * 301, 256, 256), (128 * 450, 32, 256), (128 * 333, 256, 16)])
def test_gemm_f32_matches_torch(M, N, K):
    g = torch.Generator(device=DEV).manual_seed(M * 7 + N * 3 + K)
    A = torch.randn((M, K), device=DEV, generator=g).to(torch.bfloat16)
    B = torch.randn((N, K), device=DEV, generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device=DEV, generator=g)
    C = gemm(A, B, bias)
    ref = A.float() @ B.float().T + bias
    tol = 1e-4 * (K ** 0.5) * ref.abs().max().item()
    assert (C - ref).abs().max().item() <= tol


def test_gemm_epilogues():
    M, N, K = 256, 256, 256
    g = torch.Generator(device=DEV).manual_seed(5)
    A = (0.2 * torch.randn((M, K), device=DEV, generator=g)).to(torch.bfloat16)
    B = (0.2 * torch.randn((N, K), device=DEV, generator=g)).to(torch.bfloat16)
    bias = torch.randn(N, device=DEV, generator=g)
    z = A.float() @ B.float().T + bias
    pre = torch.empty((M, N), device=DEV, dtype=torch.float32)
    y = gemm(A, B, bias, EPI_GELU, aux=pre)
    assert torch.allclose(pre, z, atol=1e-3, rtol=1e-3)
    assert torch.allclose(y.float(), gelu(z), atol=2e-2, rtol=1e-2)
    yb = gemm(A, B, bias, EPI_BF16)
    assert torch.allclose(yb.float(), z, atol=2e-2, rtol=1e-2)
    d = gemm(A, B, None, EPI_DGELU, aux=pre)
    ref = (A.float() @ B.float().T) * gelu_grad(pre)
    assert torch.allclose(d.float(), ref, atol=2e-2, rtol=1e-2)


def test_gemm_partial_columns():
    M, N, K = 128, 32, 256
    A = torch.randn((M, K), device=DEV).to(torch.bfloat16)
    B = torch.randn((N, K), device=DEV).to(torch.bfloat16)
    C = torch.full((M, N), 7.0, device=DEV)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    code = _lib.load().b200chem_mlp_gemm_bf16(A.data_ptr(), K, B.data_ptr(), K, M, N, K, C.data_ptr(), N, None, None,
                                               EPI_F32, 22, err.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert code == 0
    torch.cuda.synchronize()
    ref = A.float() @ B.float().T
    assert torch.allclose(C[:, :22], ref[:, :22], atol=1e-2, rtol=1e-3)
    assert torch.all(C[:, 22:] == 7.0)


def test_bounded_wait_times_out_and_context_survives():
    """A wait on an mbarrier that nothing completes gives up after its bound
    and raises the error flag; the next GEMM on the same context is exact."""
    import time
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    t0 = time.perf_counter()
    code = _lib.load().b200chem_selftest_bounded_wait(err.data_ptr(), 4096,
                                                      torch.cuda.current_stream().cuda_stream)
    assert code == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 1 and time.perf_counter() - t0 < 5.0
    M, N, K = 256, 256, 256
    A = torch.randn((M, K), device=DEV).to(torch.bfloat16)
    B = torch.randn((N, K), device=DEV).to(torch.bfloat16)
    C = gemm(A, B, None)
    ref = A.float() @ B.float().T
    assert (C - ref).abs().max().item() <= 1e-4 * 16 * ref.abs().max().item()


SPLIT_OUT, SPLIT_A = 0x10, 0x20


def _split(x):
    hi = x.to(torch.bfloat16)
    lo = (x - hi.float()).to(torch.bfloat16)
    return torch.cat([hi, lo], dim=1)


@pytest.mark.parametrize("M,N,K", [(256, 256, 256), (128 * 41, 32, 256), (384, 256, 32), (128, 256, 64)])
def test_two_term_operand_reaches_fp32_accuracy(M, N, K):
    """A carried as two BF16 terms (hi | lo) times BF16 B with FP32 accumulation
    matches the FP32 product of the unrounded A to ~2^-16 relative, where a
    single BF16 term is off by ~2^-9."""
    g = torch.Generator(device=DEV).manual_seed(M + N + K)
    A = torch.randn((M, K), device=DEV, generator=g)
    B = torch.randn((N, K), device=DEV, generator=g).to(torch.bfloat16)
    bias = torch.randn(N, device=DEV, generator=g)
    A2 = _split(A)
    out = torch.empty((M, N), device=DEV, dtype=torch.float32)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    code = _lib.load().b200chem_mlp_gemm_bf16(A2.data_ptr(), A2.stride(0), B.data_ptr(), B.stride(0), M, N, K,
                                               out.data_ptr(), out.stride(0), bias.data_ptr(), None,
                                               EPI_F32 | SPLIT_A, 0, err.data_ptr(),
                                               torch.cuda.current_stream().cuda_stream)
    assert code == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = A.double() @ B.double().T + bias.double()
    one = gemm(A.to(torch.bfloat16), B, bias)
    e2 = (out.double() - ref).abs().max().item()
    e1 = (one.double() - ref).abs().max().item()
    scale = (A.double().abs() @ B.double().abs().T).max().item()
    assert e2 <= 4e-5 * scale, (e2, scale)
    assert e2 < 0.1 * e1, (e2, e1)


def test_two_term_output_and_pre_activation_stride():
    """GELU epilogue written as two BF16 terms: hi + lo reproduces the FP32
    activation to ~2^-16; the pre-activations go to aux with row stride N."""
    M, N, K = 256, 256, 64
    g = torch.Generator(device=DEV).manual_seed(9)
    A = (0.3 * torch.randn((M, K), device=DEV, generator=g)).to(torch.bfloat16)
    B = (0.3 * torch.randn((N, K), device=DEV, generator=g)).to(torch.bfloat16)
    bias = 0.1 * torch.randn(N, device=DEV, generator=g)
    C = torch.empty((M, 2 * N), device=DEV, dtype=torch.bfloat16)
    pre = torch.empty((M, N), device=DEV, dtype=torch.float32)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    code = _lib.load().b200chem_mlp_gemm_bf16(A.data_ptr(), K, B.data_ptr(), K, M, N, K, C.data_ptr(), 2 * N,
                                               bias.data_ptr(), pre.data_ptr(), EPI_GELU | SPLIT_OUT, 0,
                                               err.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert code == 0
    torch.cuda.synchronize()
    z = A.float() @ B.float().T + bias
    assert torch.allclose(pre, z, atol=1e-4, rtol=1e-4)
    y = C[:, :N].float() + C[:, N:].float()
    ref = gelu(pre.double()).float()
    # tanh.approx limits the activation itself; the two-term store keeps what it computes
    assert (y - ref).abs().max().item() < 2e-3
    hi, lo = C[:, :N].float(), C[:, N:].float()
    assert torch.all(lo.abs() <= hi.abs() * 2.0 ** -8 + 1e-30)  # lo is hi's rounding residual
    assert (hi - ref).abs().mean().item() > 2.0 * (y - ref).abs().mean().item()


def test_two_term_flags_are_validated():
    M, N, K = 128, 32, 32
    A = torch.zeros((M, K), device=DEV, dtype=torch.bfloat16)
    B = torch.zeros((N, K), device=DEV, dtype=torch.bfloat16)
    C = torch.zeros((M, N), device=DEV, dtype=torch.float32)
    L = _lib.load()
    st = torch.cuda.current_stream().cuda_stream
    # lda too small for two terms
    assert L.b200chem_mlp_gemm_bf16(A.data_ptr(), K, B.data_ptr(), K, M, N, K, C.data_ptr(), N, None, None,
                                    EPI_F32 | SPLIT_A, 0, None, st) == -1
    # two-term output needs a BF16 epilogue and ldc >= 2N
    assert L.b200chem_mlp_gemm_bf16(A.data_ptr(), K, B.data_ptr(), K, M, N, K, C.data_ptr(), N, None, None,
                                    EPI_F32 | SPLIT_OUT, 0, None, st) == -1


def test_fused_adam_matches_reference_update():
    rows, cols = 48, 40
    g = torch.Generator(device=DEV).manual_seed(3)
    p = torch.randn((rows, cols), device=DEV, generator=g)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    pr, mr, vr = p.clone(), m.clone(), v.clone()
    wb = torch.empty((rows, cols), device=DEV, dtype=torch.bfloat16)
    wbt = torch.empty((cols, rows), device=DEV, dtype=torch.bfloat16)
    L = _lib.load()
    for step in range(1, 4):
        grad = torch.randn((rows, cols), device=DEV, generator=g)
        code = L.b200chem_mlp_adam(p.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(), rows, cols, 1e-2,
                                   0.9, 0.999, 1e-8, step, wb.data_ptr(), wbt.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream)
        assert code == 0
        mr = 0.9 * mr + 0.1 * grad
        vr = 0.999 * vr + 0.001 * grad * grad
        pr = pr - 1e-2 * (mr / (1 - 0.9 ** step)) / ((vr / (1 - 0.999 ** step)).sqrt() + 1e-8)
    torch.cuda.synchronize()
    assert torch.allclose(p, pr, rtol=1e-5, atol=1e-6)
    assert torch.equal(wb, p.to(torch.bfloat16)) and torch.equal(wbt, p.t().to(torch.bfloat16))
