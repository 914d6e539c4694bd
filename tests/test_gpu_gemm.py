"""tcgen05 BF16 GEMM against a plain PyTorch fp32 reference of the same op
(fp32 matmul of the same bf16 values).  Tolerance (written here): fp32 output
within 1e-5 * sqrt(K) * max|C| + 1e-6 (summation order only); bf16 output
within one bf16 ulp (2^-8 relative) of the rounded reference."""
import math

import pytest

pytestmark = pytest.mark.gpu


def _ref(A, B, bias, relu, mask):
    C = A.float() @ B.float().T
    if bias is not None:
        C = C + bias
    if relu:
        C = C.clamp_min(0)
    if mask is not None:
        C = C * (mask.float() > 0)
    return C


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 1024), (200, 130, 72), (1000, 2652, 1024),
                                   (512, 1024, 2752), (7, 9, 8)])
def test_gemm_fp32_out(mtt, cuda, M, N, K):
    import torch
    g = torch.Generator(device="cpu").manual_seed(M * 31 + N)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).to(cuda)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).to(cuda)
    C = mtt.gemm_bf16(A, B)
    R = _ref(A, B, None, False, None)
    tol = 1e-5 * math.sqrt(K) * float(R.abs().max()) + 1e-6
    assert float((C - R).abs().max()) <= tol


def test_gemm_bias_relu_bf16_and_mask(mtt, cuda):
    import torch
    g = torch.Generator(device="cpu").manual_seed(5)
    M, N, K = 384, 256, 512
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).to(cuda)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).to(cuda)
    bias = torch.randn(N, generator=g).to(cuda)
    C = mtt.gemm_bf16(A, B, bias=bias, relu=True, out_bf16=True)
    R = _ref(A, B, bias, True, None)
    assert C.dtype == torch.bfloat16
    assert float(((C.float() - R).abs() / (R.abs() + 1e-3)).max()) <= 2 ** -8 + 1e-6
    mask = torch.randn(M, N, generator=g).to(torch.bfloat16).to(cuda)
    C2 = mtt.gemm_bf16(A, B, mask=mask)
    R2 = _ref(A, B, None, False, mask)
    assert float((C2 - R2).abs().max()) <= 1e-5 * math.sqrt(K) * float(R2.abs().max()) + 1e-6
    assert bool((C2[mask.float() <= 0] == 0).all())


def test_gemm_strided_operands(mtt, cuda):
    """Row strides larger than K (views into wider buffers) and an output
    written into a wider matrix."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(9)
    Abig = torch.randn(300, 200, generator=g).to(torch.bfloat16).to(cuda)
    Bbig = torch.randn(140, 136, generator=g).to(torch.bfloat16).to(cuda)
    A, B = Abig[:, :128], Bbig[:, :128]
    out = torch.zeros(300, 160, device=cuda)
    mtt.gemm_bf16(A, B, out=out[:, :140])
    R = _ref(A, B, None, False, None)
    assert float((out[:, :140] - R).abs().max()) <= 1e-5 * math.sqrt(128) * float(R.abs().max()) + 1e-6
    assert float(out[:, 140:].abs().max()) == 0.0


@pytest.mark.parametrize("M,N,K,relu,out_bf16,masked", [
    (240, 1024, 2752, True, True, False),     # the leaf network's first layer at 5 leaves x 48 rivers
    (240, 2688, 1024, False, False, False),   # its output layer
    (1024, 1024, 4096, False, False, False),  # a weight gradient of the training step
    (200, 130, 1000, False, False, True),     # ragged edges, a ReLU mask
])
def test_split_k_workspace_matches_reference_and_one_pass(mtt, cuda, M, N, K, relu, out_bf16, masked):
    """mtt_gemm_bf16_ws: few output tiles over a long K are split along K
    into a workspace and added in split order.  Same tolerance as above
    against the fp32 reference; deterministic (two calls agree bit for bit);
    a workspace too small for any split gives the one-pass kernel's bits."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(M + 7 * N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).to(cuda)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).to(cuda)
    bias = torch.randn(N, generator=g).to(cuda)
    mask = torch.randn(M, N, generator=g).to(torch.bfloat16).to(cuda) if masked else None
    ws = torch.empty(16 * M * N, dtype=torch.float32, device=cuda)
    kw = dict(bias=bias, relu=relu, out_bf16=out_bf16, mask=mask)
    C1 = mtt.gemm_bf16(A, B, workspace=ws, **kw)
    C2 = mtt.gemm_bf16(A, B, workspace=ws, **kw)
    assert torch.equal(C1, C2)
    R = _ref(A, B, bias, relu, mask)
    tol = 1e-5 * math.sqrt(K) * float(R.abs().max()) + 1e-6       # FP32 summation order
    if out_bf16:   # plus one bf16 rounding of the FP32 result
        assert bool(((C1.float() - R).abs() <= 2 ** -8 * R.abs() + tol).all())
    else:
        assert float((C1.float() - R).abs().max()) <= tol
    one = mtt.gemm_bf16(A, B, **kw)
    tiny = mtt.gemm_bf16(A, B, workspace=ws[: M * N], **kw)   # room for one split only: no split
    assert torch.equal(tiny, one)
