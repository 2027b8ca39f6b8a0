"""The learned smoother's CPU restatement (oracle/conv.c), pinned on its own
mathematics before the tensor-core kernels are compared against it (CPU only).

There is no reference counterpart for the conv net, so the oracle is checked
by properties: BF16 rounding against an independent vectorised rounding,
the transposed convolution as the exact adjoint of the convolution, the
weight gradient as the bilinear derivative, and the whole-network loss
gradient against central finite differences in FP32 mode.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _rand_weights(rng, ci_used=16, co_used=16, scale=0.2):
    w = np.zeros((27, 16, 16), np.float32)
    w[:, :ci_used, :co_used] = rng.standard_normal((27, ci_used, co_used)).astype(np.float32) * scale
    return w.reshape(-1)


def test_bf16_rounding_matches_vectorised():
    rng = np.random.default_rng(1)
    v = np.concatenate([rng.standard_normal(2000).astype(np.float32) * 10.0 ** rng.integers(-20, 20, 2000),
                        np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.0e38, -3.0e38], np.float32)])
    L = O.colored_lib()
    scalar = np.array([L.oc_bf16(float(x)) for x in v], np.float32)
    assert np.array_equal(scalar.view(np.uint32), O.bf16(v).view(np.uint32))
    # ties go to even: 1 + 2^-8 sits halfway between 1 and 1 + 2^-7
    assert O.bf16(np.array([1.00390625], np.float32))[0] == 1.0
    assert O.bf16(np.array([1.01171875], np.float32))[0] == 1.015625


def test_conv_identity_tap():
    # a weight that is the identity on the centre tap copies the input
    dims = (3, 4, 5)
    n = 60
    rng = np.random.default_rng(2)
    x = rng.standard_normal(n * 16).astype(np.float32)
    w = np.zeros((27, 16, 16), np.float32)
    w[13] = np.eye(16)
    y = O.conv16(dims, x, w.reshape(-1), round_=False)
    assert np.array_equal(y, x)


def test_transposed_conv_is_adjoint():
    dims = (4, 5, 6)
    n = 120
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n * 16).astype(np.float32)
    g = rng.standard_normal(n * 16).astype(np.float32)
    w = _rand_weights(rng)
    lhs = np.dot(O.conv16(dims, x, w, round_=False).astype(np.float64), g)
    rhs = np.dot(x.astype(np.float64), O.conv16(dims, g, O.flip_transpose(w), round_=False))
    assert abs(lhs - rhs) <= 1e-4 * (abs(lhs) + 1.0)


def test_wgrad_is_bilinear_derivative():
    # <conv(x, W), g> is linear in W with gradient wgrad(x, g)
    dims = (4, 5, 6)
    n = 120
    rng = np.random.default_rng(4)
    x = rng.standard_normal(n * 16).astype(np.float32)
    g = rng.standard_normal(n * 16).astype(np.float32)
    w = _rand_weights(rng)
    dw = O.conv16_wgrad(dims, x, g, round_=False)
    f = np.dot(O.conv16(dims, x, w, round_=False).astype(np.float64), g)
    assert abs(f - np.dot(dw.astype(np.float64), w)) <= 1e-4 * (abs(f) + 1.0)


@pytest.mark.parametrize("odd,kind", [(False, 0), (True, 0), (False, 1), (True, 1)])
def test_net_gradient_finite_differences(odd, kind):
    dims = (5, 4, 6)
    n = 120
    rng = np.random.default_rng(5)
    w1 = _rand_weights(rng, ci_used=1, scale=0.5)
    w2 = _rand_weights(rng, scale=0.15)
    w3 = _rand_weights(rng, co_used=1, scale=0.15)
    r = rng.standard_normal(n).astype(np.float32)
    e = rng.standard_normal(n).astype(np.float32)
    loss, grads = O.net_loss_grad(dims, w1, w2, w3, r, e, round_=False, odd=odd, kind=kind)
    ws = [w1, w2, w3]
    used = [np.nonzero(w1)[0], np.nonzero(w2)[0], np.nonzero(w3)[0]]
    h = 3e-3
    rel = []
    for layer in range(3):
        for idx in rng.choice(used[layer], 8, replace=False):
            wp = [w.copy() for w in ws]
            wm = [w.copy() for w in ws]
            wp[layer][idx] += h
            wm[layer][idx] -= h
            lp, _ = O.net_loss_grad(dims, *wp, r, e, round_=False, odd=odd, kind=kind)
            lm, _ = O.net_loss_grad(dims, *wm, r, e, round_=False, odd=odd, kind=kind)
            fd = (lp - lm) / (2 * h)
            rel.append(abs(fd - float(grads[layer][idx])) / max(abs(fd), 1e-3))
    # the net is piecewise linear: a step that crosses a ReLU kink spoils a
    # few differences, the bulk must agree closely
    rel = np.array(rel)
    assert np.median(rel) < 2e-3, rel
    assert np.mean(rel < 1e-2) >= 0.8, rel
    assert rel.max() < 0.2, rel
    assert loss > 0


def test_net_bf16_close_to_fp32():
    dims = (6, 6, 6)
    n = 216
    rng = np.random.default_rng(6)
    w1 = _rand_weights(rng, ci_used=1, scale=0.5)
    w2 = _rand_weights(rng, scale=0.15)
    w3 = _rand_weights(rng, co_used=1, scale=0.15)
    r = rng.standard_normal(n).astype(np.float32)
    y32, _, _ = O.net_forward(dims, w1, w2, w3, r, round_=False)
    y16, a1, _ = O.net_forward(dims, w1, w2, w3, r, round_=True)
    assert np.array_equal(a1, O.bf16(a1))  # hidden activations are stored as bf16
    assert np.linalg.norm(y16 - y32) <= 2e-2 * np.linalg.norm(y32)


def test_odd_network_is_odd_and_energy_loss_matches_definition():
    dims = (4, 5, 6)
    n = 120
    rng = np.random.default_rng(8)
    w1 = _rand_weights(rng, ci_used=1, scale=0.5)
    w2 = _rand_weights(rng, scale=0.15)
    w3 = _rand_weights(rng, co_used=1, scale=0.15)
    r = rng.standard_normal(n).astype(np.float32)
    e = rng.standard_normal(n).astype(np.float32)
    yp = O.net_forward(dims, w1, w2, w3, r, round_=False)[0]
    ym = O.net_forward(dims, w1, w2, w3, -r, round_=False)[0]
    y = 0.5 * (yp - ym)
    d = (y - e).astype(np.float32)
    want = np.dot(d.astype(np.float64), O.stencil_apply(dims, d)) / np.dot(e.astype(np.float64),
                                                                           O.stencil_apply(dims, e))
    loss, _ = O.net_loss_grad(dims, w1, w2, w3, r, e, round_=False, odd=True, kind=1)
    assert abs(loss - want) <= 1e-5 * want
    # the stencil is the HPCG matrix: symmetric, diagonal 26
    v = rng.standard_normal(n).astype(np.float32)
    assert abs(np.dot(O.stencil_apply(dims, v), e) - np.dot(v, O.stencil_apply(dims, e))) < 1e-3
