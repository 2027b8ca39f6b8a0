"""hpcgb200_dot_noalloc: the dot product for callers that cannot allocate
device memory (their device memory belongs to their own pool, or cudaMalloc's
possible device synchronization is not allowed on their path).  It takes no
workspace: its scratch is a fixed array inside the library.  Checked through
the C ABI against hpcgb200_dot (the workspace version) and against an FP64
sum on the host, on two calls in a row, with the tolerance the other
dot-product tests use; two launches queued without a host synchronization in
between exercise the hand-over of the shared scratch; sizes above its stated
maximum must be rejected.  Kept in its own file, collected last."""
import ctypes
import math

import pytest
import torch

import rochpcg_b200 as R

pytestmark = pytest.mark.gpu

MAX_N = 4096 * 4096  # stated maximum of hpcgb200_dot_noalloc


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def reference_dot(L, x, y, s):
    nb = L.hpcgb200_reduction_workspace_bytes()
    ws = torch.zeros(nb, dtype=torch.uint8, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert L.hpcgb200_dot(x.numel(), vp(x), vp(y), vp(out), vp(ws), nb, s) == 0
    return out


def host_dot(x, y):
    """FP64 sum on the host of the products (each product rounded to FP64,
    the sum correctly rounded)."""
    return math.fsum((x.cpu().numpy() * y.cpu().numpy()).tolist())


def close(a, b, x, y):
    scale = max(1.0, float((x.abs() * y.abs()).sum()))
    return abs(a - b) <= 1e-12 * scale


@pytest.mark.parametrize("n", [1, 4097, 3_000_001, 4096 * 4095 + 1, MAX_N - 1, MAX_N])
def test_noalloc_dot_two_calls_match_workspace_dot(n):
    L = R.load()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(n)
    res = []
    for call in range(2):  # two calls in a row share the library's scratch
        x = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - 0.5
        y = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - 0.5
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        assert L.hpcgb200_dot_noalloc(n, vp(x), vp(y), vp(out), s) == 0, L.hpcgb200_last_error()
        ref = reference_dot(L, x, y, s)
        torch.cuda.synchronize()
        assert close(out.item(), ref.item(), x, y)
        assert close(out.item(), host_dot(x, y), x, y)
        res.append(out.item())
    assert res[0] != res[1]


@pytest.mark.parametrize("n", [4096 * 7 + 5, MAX_N])
def test_noalloc_dot_back_to_back_without_host_sync(n):
    """Two launches queued on one stream with no synchronization between them:
    the second must find the scratch's ticket handed back by the first."""
    L = R.load()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(n + 1)
    xs = [torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - 0.5 for _ in range(2)]
    ys = [torch.rand(n, dtype=torch.float64, device="cuda", generator=g) - 0.5 for _ in range(2)]
    outs = [torch.full((1,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    for k in range(2):
        assert L.hpcgb200_dot_noalloc(n, vp(xs[k]), vp(ys[k]), vp(outs[k]), s) == 0, L.hpcgb200_last_error()
    torch.cuda.synchronize()
    for k in range(2):
        assert close(outs[k].item(), host_dot(xs[k], ys[k]), xs[k], ys[k])
    # a third call on the first pair reproduces the first result bit for bit
    again = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    assert L.hpcgb200_dot_noalloc(n, vp(xs[0]), vp(ys[0]), vp(again), s) == 0
    torch.cuda.synchronize()
    assert again.item() == outs[0].item()


def test_noalloc_dot_rejects_sizes_above_maximum():
    L = R.load()
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.hpcgb200_dot_noalloc(MAX_N + 1, vp(x), vp(x), vp(out), s) == 1
    assert b"exceeds" in L.hpcgb200_last_error()
    assert L.hpcgb200_dot_noalloc(0, vp(x), vp(x), vp(out), s) == 0
    torch.cuda.synchronize()
    assert out.item() == 0.0
