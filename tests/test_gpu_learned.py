"""Learned-smoother tensor-core kernels against the conv-net oracle
(oracle/conv.c): forward convolution in every epilogue, the transposed
convolution, and the weight gradient, on ragged grids and batches.

Tolerances: inputs and weights are the same BF16 values on both sides and
both accumulate in FP32, so the sums differ only by summation order
(|err| <= 1e-5 of sum |a||w|); BF16 outputs may differ by one BF16 ulp when
that order moves a value across a rounding boundary.
"""
import ctypes

import numpy as np
import pytest
import torch

import rochpcg_b200 as R
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RELU, MASK, F32, F32C0 = 0, 1, 2, 3


def vp(t):
    return ctypes.c_void_p(t.data_ptr())


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def bf16_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(torch.bfloat16).cuda()


def rand_weights(rng, scale=0.3):
    return O.bf16(rng.standard_normal(27 * 256).astype(np.float32) * scale)


def prepared(w, flip=0):
    L = R.load()
    wd = torch.from_numpy(w).cuda()
    wB = torch.empty(L.hpcgb200_conv_weight_tile_bytes(), dtype=torch.uint8, device="cuda")
    assert L.hpcgb200_conv_prepare_weights(vp(wd), vp(wB), flip, stream()) == 0
    return wB


def conv_dev(dims, nb, x, wB, mode, act=None):
    L = R.load()
    nz, ny, nx = dims
    n = nb * nz * ny * nx
    if mode in (RELU, MASK):
        out = torch.empty(n * 16, dtype=torch.bfloat16, device="cuda")
    elif mode == F32:
        out = torch.empty(n * 16, dtype=torch.float32, device="cuda")
    else:
        out = torch.empty(n, dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.hpcgb200_conv16(nb, nz, ny, nx, vp(x), vp(wB), mode, vp(out), vp(act) if act is not None else None,
                           vp(status), stream())
    assert rc == 0, L.hpcgb200_last_error()
    torch.cuda.synchronize()
    assert status.item() == 0
    return out.float().cpu().numpy()


def oracle_conv(dims, nb, x, w):
    per = int(np.prod(dims)) * 16
    return np.concatenate([O.conv16(dims, x[b * per:(b + 1) * per], w, round_=False) for b in range(nb)])


def abs_bound(dims, nb, x, w):
    return oracle_conv(dims, nb, np.abs(x), np.abs(w))


# (z, y, x) extents: partial bricks in every dimension, x across the 14-point
# brick stride (16, 20, 33, 40) and on it (14, 28)
GRIDS = [((2, 8, 16), 1), ((5, 12, 20), 3), ((3, 3, 3), 2), ((1, 1, 40), 1), ((16, 16, 16), 2), ((9, 17, 33), 1),
         ((4, 8, 28), 2), ((6, 10, 14), 1)]


@pytest.mark.parametrize("dims,nb", GRIDS)
def test_conv_forward_f32(dims, nb):
    rng = np.random.default_rng(sum(dims) + nb)
    n = nb * int(np.prod(dims))
    x = O.bf16(rng.standard_normal(n * 16).astype(np.float32))
    w = rand_weights(rng)
    got = conv_dev(dims, nb, bf16_dev(x), prepared(w), F32)
    ref = oracle_conv(dims, nb, x, w)
    bound = abs_bound(dims, nb, x, w)
    assert np.all(np.abs(got - ref) <= 1e-5 * bound + 1e-30)
    # channel 0 only
    got0 = conv_dev(dims, nb, bf16_dev(x), prepared(w), F32C0)
    assert np.array_equal(got0, got[0::16])


@pytest.mark.parametrize("dims,nb", GRIDS[:3])
def test_conv_relu_and_mask_epilogues(dims, nb):
    rng = np.random.default_rng(7 + nb)
    n = nb * int(np.prod(dims))
    x = O.bf16(rng.standard_normal(n * 16).astype(np.float32))
    w = rand_weights(rng)
    ref = oracle_conv(dims, nb, x, w)
    got = conv_dev(dims, nb, bf16_dev(x), prepared(w), RELU)
    want = O.bf16(np.maximum(ref, 0.0))
    ulp = np.abs(want) * 2.0 ** -7 + 1e-30
    assert np.all(np.abs(got - want) <= ulp)
    assert np.mean(got == want) > 0.99
    # mask by an activation tensor: keeps the conv where act > 0
    act = O.bf16(rng.standard_normal(n * 16).astype(np.float32))
    gotm = conv_dev(dims, nb, bf16_dev(x), prepared(w), MASK, act=bf16_dev(act))
    wantm = O.bf16(np.where(act > 0, ref, 0.0).astype(np.float32))
    assert np.all(np.abs(gotm - wantm) <= np.abs(wantm) * 2.0 ** -7 + 1e-30)
    assert np.all(gotm[act <= 0] == 0)


@pytest.mark.parametrize("dims,nb", [((5, 12, 20), 2), ((16, 16, 16), 1)])
def test_transposed_conv(dims, nb):
    rng = np.random.default_rng(11)
    n = nb * int(np.prod(dims))
    g = O.bf16(rng.standard_normal(n * 16).astype(np.float32))
    w = rand_weights(rng)
    got = conv_dev(dims, nb, bf16_dev(g), prepared(w, flip=1), F32)
    wt = O.flip_transpose(w)
    ref = oracle_conv(dims, nb, g, wt)
    assert np.all(np.abs(got - ref) <= 1e-5 * abs_bound(dims, nb, g, wt) + 1e-30)


@pytest.mark.parametrize("dims,nb", [((2, 8, 16), 1), ((5, 12, 20), 3), ((16, 16, 16), 4), ((7, 9, 11), 2)])
def test_weight_gradient(dims, nb):
    L = R.load()
    rng = np.random.default_rng(13 + nb)
    nz, ny, nx = dims
    per = nz * ny * nx
    n = nb * per
    x = O.bf16(rng.standard_normal(n * 16).astype(np.float32))
    g = O.bf16(rng.standard_normal(n * 16).astype(np.float32))
    partial = torch.empty(L.hpcgb200_conv_wgrad_partial_bytes(nb, nz, ny, nx) // 4, dtype=torch.float32,
                          device="cuda")
    dw = torch.empty(27 * 256, dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.hpcgb200_conv16_wgrad(nb, nz, ny, nx, vp(bf16_dev(x)), vp(bf16_dev(g)), vp(partial), vp(dw),
                                   vp(status), stream()) == 0
    torch.cuda.synchronize()
    assert status.item() == 0
    got = dw.cpu().numpy()
    ref = sum(O.conv16_wgrad(dims, x[b * per * 16:(b + 1) * per * 16], g[b * per * 16:(b + 1) * per * 16],
                             round_=False) for b in range(nb))
    bound = sum(O.conv16_wgrad(dims, np.abs(x[b * per * 16:(b + 1) * per * 16]),
                               np.abs(g[b * per * 16:(b + 1) * per * 16]), round_=False) for b in range(nb))
    assert np.all(np.abs(got - ref) <= 2e-5 * bound + 1e-30)
    # deterministic: a second launch gives the same bits
    dw2 = torch.empty_like(dw)
    assert L.hpcgb200_conv16_wgrad(nb, nz, ny, nx, vp(bf16_dev(x)), vp(bf16_dev(g)), vp(partial), vp(dw2),
                                   vp(status), stream()) == 0
    torch.cuda.synchronize()
    assert torch.equal(dw, dw2)


def test_conv_argument_errors():
    L = R.load()
    x = torch.zeros(16, dtype=torch.bfloat16, device="cuda")
    wB = torch.zeros(L.hpcgb200_conv_weight_tile_bytes(), dtype=torch.uint8, device="cuda")
    out = torch.zeros(16, dtype=torch.float32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert L.hpcgb200_conv16(1, 1, 1, 1, vp(x), vp(wB), 9, vp(out), None, vp(st), stream()) != 0
    assert L.hpcgb200_conv16(1, 1, 1, 1, vp(x), vp(wB), MASK, vp(out), None, vp(st), stream()) != 0
    assert L.hpcgb200_conv16(0, 1, 1, 1, vp(x), vp(wB), F32, vp(out), None, vp(st), stream()) != 0
