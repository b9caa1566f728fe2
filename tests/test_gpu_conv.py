"""Tensor-core (tcgen05) kernels of the warm-start network against plain
PyTorch FP32 references of the same ops, on BF16-rounded inputs.

Tolerances: GEMM (FP32 accumulate, FP32 output) 1e-4 of max |ref|;
convolutions (FP32 accumulate, BF16 output) 1e-2 of max |ref| (BF16 keeps 8
mantissa bits)."""
import ctypes

import pytest
import torch
import torch.nn.functional as F


def _tc_ok(nat):
    e = ctypes.c_int(0)
    nat.check(nat.lib().fem_tc_error(ctypes.byref(e), 1), "tc_error")
    assert e.value == 0, f"tensor-core pipeline timeout code {e.value}"


@pytest.mark.gpu
@pytest.mark.parametrize("M,N,K,split", [(300, 64, 432, 1), (256, 128, 1024, 4), (200, 32, 96, 3),
                                         (129, 16, 160, 2), (512, 256, 512, 2)])
def test_gemm_tn(pkg, cuda, M, N, K, split):
    nat = pkg._native
    g = torch.Generator(device="cpu").manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).to(cuda, torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(cuda, torch.bfloat16)
    C = torch.zeros(M, N, dtype=torch.float32, device=cuda)
    nat.check(nat.lib().fem_gemm_bf16_tn_f32(nat.ptr(A), nat.ptr(B), nat.ptr(C), M, N, K, N, split,
                                             nat.stream_ptr()), "gemm")
    torch.cuda.synchronize()
    _tc_ok(nat)
    ref = A.float() @ B.float().T
    assert (C - ref).abs().max().item() <= 1e-4 * ref.abs().max().item()


def _conv(nat, x, w, b, relu):
    N, D, H, W, Cin = x.shape
    Cout = w.shape[0]
    out = torch.empty(N, D, H, W, Cout, dtype=torch.bfloat16, device=x.device)
    nat.check(nat.lib().fem_conv3d_fwd_bf16(nat.ptr(x), nat.ptr(w), nat.ptr(b), nat.ptr(out), N, D, H, W, Cin,
                                            Cout, int(relu), nat.stream_ptr()), "conv3d")
    return out


def _torch_conv(x, w, b, relu):
    # x NDHWC, w (Cout, 27, Cin) -> torch (Cout, Cin, 3, 3, 3)
    Cout, _, Cin = w.shape
    wt = w.float().reshape(Cout, 3, 3, 3, Cin).permute(0, 4, 1, 2, 3)
    y = F.conv3d(x.float().permute(0, 4, 1, 2, 3), wt, None if b is None else b.float(), padding=1)
    if relu:
        y = torch.relu(y)
    return y.permute(0, 2, 3, 4, 1)


SHAPES = [(2, 8, 16, 16, 16, 32), (8, 4, 2, 2, 64, 128), (2, 16, 8, 8, 32, 16), (1, 4, 4, 8, 128, 64),
          (4, 8, 4, 4, 16, 16)]


@pytest.mark.gpu
@pytest.mark.parametrize("N,D,H,W,Cin,Cout", SHAPES)
def test_conv3d_fwd(pkg, cuda, N, D, H, W, Cin, Cout):
    nat = pkg._native
    g = torch.Generator(device="cpu").manual_seed(Cin * 7 + Cout)
    x = torch.randn(N, D, H, W, Cin, generator=g).to(cuda, torch.bfloat16)
    w = (torch.randn(Cout, 27, Cin, generator=g) / (27 * Cin) ** 0.5).to(cuda, torch.bfloat16)
    b = torch.randn(Cout, generator=g).to(cuda)
    for relu in (False, True):
        y = _conv(nat, x, w, b, relu)
        torch.cuda.synchronize()
        _tc_ok(nat)
        ref = _torch_conv(x, w, b, relu)
        assert (y.float() - ref).abs().max().item() <= 1e-2 * ref.abs().max().item()


@pytest.mark.gpu
@pytest.mark.parametrize("N,D,H,W,Cin,Cout", SHAPES[:3])
def test_conv3d_backward(pkg, cuda, N, D, H, W, Cin, Cout):
    nat = pkg._native
    g = torch.Generator(device="cpu").manual_seed(5 + Cin)
    x = torch.randn(N, D, H, W, Cin, generator=g).to(cuda, torch.bfloat16)
    w = (torch.randn(Cout, 27, Cin, generator=g) / (27 * Cin) ** 0.5).to(cuda, torch.bfloat16)
    dy = torch.randn(N, D, H, W, Cout, generator=g).to(cuda, torch.bfloat16)
    # reference gradients in FP32
    xr = x.float().requires_grad_(True)
    wr = w.float().requires_grad_(True)
    y = _torch_conv(xr, wr, None, False)
    y.backward(dy.float())
    # dgrad: conv of dy with flipped, transposed weights
    wt = torch.empty(Cin, 27, Cout, dtype=torch.bfloat16, device=cuda)
    nat.check(nat.lib().fem_conv3d_flip_weights_bf16(nat.ptr(w), nat.ptr(wt), Cout, Cin, nat.stream_ptr()), "flip")
    if Cin in (16, 32, 64, 128):
        dx = _conv(nat, dy, wt, None, False)
        torch.cuda.synchronize()
        _tc_ok(nat)
        assert (dx.float() - xr.grad).abs().max().item() <= 1e-2 * xr.grad.abs().max().item()
    # wgrad: dW^T = im2col(x)^T dz
    V = N * D * H * W
    col = torch.empty(27 * Cin, V, dtype=torch.bfloat16, device=cuda)
    nat.check(nat.lib().fem_conv3d_im2col_t_bf16(nat.ptr(x), nat.ptr(col), N, D, H, W, Cin, nat.stream_ptr()),
              "im2col")
    dyt = torch.empty(Cout, V, dtype=torch.bfloat16, device=cuda)
    nat.check(nat.lib().fem_transpose_bf16(nat.ptr(dy), nat.ptr(dyt), V, Cout, nat.stream_ptr()), "transpose")
    dwt = torch.zeros(27 * Cin, Cout, dtype=torch.float32, device=cuda)
    nat.check(nat.lib().fem_gemm_bf16_tn_f32(nat.ptr(col), nat.ptr(dyt), nat.ptr(dwt), 27 * Cin, Cout, V, Cout,
                                             8, nat.stream_ptr()), "wgrad")
    torch.cuda.synchronize()
    _tc_ok(nat)
    dw = dwt.reshape(27, Cin, Cout).permute(2, 0, 1)  # (Cout, 27, Cin)
    assert (dw - wr.grad).abs().max().item() <= 1e-3 * wr.grad.abs().max().item()
