"""CPU restatement of the tcgen05 network kernels' issue plans and data
layouts (rochpcg_b200/csrc/learned.cu).  k_conv16: the weight slot order, the
MMAs per (staged plane, row shift) with the dz and dx taps stacked in N, their
accumulate flags, the shared-memory and TMEM ranges they touch, and the
epilogue's combination of the dx blocks of neighbouring rows -- checked
exhaustively for brick depths 1-5 and numerically against a direct 3x3x3
convolution of one brick.  k_layer3_tc: taps stacked in N, the odd pair folded
into K, the 27-term gather.  k_layer1_tc: the im2col layout and product."""
import numpy as np
import pytest

KTX, KTY = 16, 8          # staged x width (14 outputs + halo), output y
KHY = KTY + 2
CH = 16
PLANE_COLS = 3 * CH       # TMEM columns of one output plane: 3 dx blocks x 16 channels
TILE = CH * CH * 2        # bytes of one tap's 16 x 16 BF16 weight tile
TMEM_COLS = 512


def weight_slot(t):
    """Tile slot of tap t = (dz+1)*9 + (dy+1)*3 + (dx+1): [dy][dz = +1, 0, -1][dx]."""
    return ((t // 3) % 3) * 9 + (2 - t // 9) * 3 + t % 3


def plan(ktz):
    """(plane q, row shift dyi, first output plane, last output plane, accumulate)."""
    for q in range(ktz + 2):
        lo, hi = max(q - 2, 0), min(q, ktz - 1)
        for dyi in range(3):
            if q <= ktz - 1 and dyi == 0:
                if hi > lo:
                    yield q, dyi, lo, hi - 1, 1
                yield q, dyi, hi, hi, 0
            else:
                yield q, dyi, lo, hi, 1


def test_weight_slots_are_a_permutation_in_dy_dz_dx_order():
    slots = [weight_slot(t) for t in range(27)]
    assert sorted(slots) == list(range(27))
    for t in range(27):
        dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
        assert weight_slot(t) == (dy + 1) * 9 + (1 - dz) * 3 + (dx + 1)


@pytest.mark.parametrize("ktz", [1, 2, 3, 4, 5])
def test_plan_covers_every_tap_once(ktz):
    touched, cover, n = set(), set(), 0
    for q, dyi, m0, m1, acc in plan(ktz):
        n += 1
        N = (m1 - m0 + 1) * PLANE_COLS
        assert N % 16 == 0 and 16 <= N <= 256                         # kind::f16 with M = 128
        b_off = dyi * 9 * TILE + (m0 - q + 2) * 3 * TILE
        assert 0 <= b_off and b_off + N * 2 * CH <= 27 * TILE          # inside the weight tiles
        assert (q * KHY + dyi) * KTX + 128 <= KTX * KHY * (ktz + 2)   # A rows inside the staged box
        for a in (0, 1):                                               # both accumulators
            assert a * ktz * PLANE_COLS + (m1 + 1) * PLANE_COLS <= TMEM_COLS
        for mt in range(m0, m1 + 1):
            dz = 1 - (mt - q + 2)
            assert dz in (-1, 0, 1) and q == mt + 1 + dz
            assert (mt in touched) == (acc == 1)                       # first write clears, later ones add
            touched.add(mt)
            for dx in (-1, 0, 1):
                key = (mt, dz, dyi - 1, dx)
                assert key not in cover
                cover.add(key)
    assert len(cover) == 27 * ktz
    assert n == 3 * (ktz + 2) + ktz - 1                                # 21 for ktz = 4


@pytest.mark.parametrize("ktz", [1, 4])
def test_plan_and_epilogue_equal_a_direct_convolution(ktz):
    rng = np.random.default_rng(ktz)
    box = rng.standard_normal((ktz + 2, KHY, KTX, CH))                 # staged [z][y][x][ci], halo included
    w = rng.standard_normal((27, CH, CH))                              # w[tap][ci][co]
    # B operand rows: slot * 16 + co, K = ci
    B = np.zeros((27 * CH, CH))
    for t in range(27):
        B[weight_slot(t) * CH:(weight_slot(t) + 1) * CH, :] = w[t].T
    D = np.zeros((128, ktz * PLANE_COLS))
    for q, dyi, m0, m1, acc in plan(ktz):
        A = box[q, dyi:dyi + KTY, :, :].reshape(128, CH)               # row m = y * 16 + x of the shifted plane
        r0 = (dyi * 9 + (m0 - q + 2) * 3) * CH
        nrows = (m1 - m0 + 1) * PLANE_COLS
        prod = A @ B[r0:r0 + nrows].T
        cols = slice(m0 * PLANE_COLS, m0 * PLANE_COLS + nrows)
        D[:, cols] = prod if acc == 0 else D[:, cols] + prod
    for mt in range(ktz):
        blk = D[:, mt * PLANE_COLS:(mt + 1) * PLANE_COLS].reshape(KTY, KTX, 3, CH)
        # out(x) = D_{dx=-1}[x - 1] + D_{dx=0}[x] + D_{dx=+1}[x + 1] for the 14 inner columns
        got = blk[:, 0:14, 0] + blk[:, 1:15, 1] + blk[:, 2:16, 2]
        want = np.zeros((KTY, 14, CH))
        for t in range(27):
            dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
            src = box[mt + 1 + dz, 1 + dy:1 + dy + KTY, 1 + dx:1 + dx + 14, :]
            want += src @ w[t]
        assert np.allclose(got, want, rtol=1e-12, atol=1e-12)


# ---- the one-channel layers (k_layer3_tc, k_layer1_tc)

K3X, K3Y, K3Z = 16, 8, 2                     # layer-3 output brick
K3HX, K3HY, K3HZ = K3X + 2, K3Y + 2, K3Z + 2  # its staged box, 720 points
K3N = 32                                      # 27 taps + 5 zero columns


def test_layer3_tap_stacking_and_pair_folding_equal_the_odd_conv():
    """D[p][t] = sum_c a[p][c] w[t][c] over the staged points (pair folded into
    K with the weights halved and negated), then y[o] = sum_t D[o + off_t][t]
    in tap order, equals (conv(a+) - conv(a-)) / 2 on the brick's outputs."""
    rng = np.random.default_rng(3)
    rows = K3HX * K3HY * K3HZ
    chunks = (rows + 127) // 128
    assert chunks * 128 >= rows and chunks * K3N * 2 <= 512          # two accumulators fit TMEM
    pos = rng.standard_normal((K3HZ, K3HY, K3HX, CH))
    neg = rng.standard_normal((K3HZ, K3HY, K3HX, CH))
    w = rng.standard_normal((27, CH))                               # w3[t][ci][0]
    B = np.zeros((K3N, CH))
    B[:27] = 0.5 * w
    D = pos.reshape(rows, CH) @ B.T + neg.reshape(rows, CH) @ (-B).T
    got = np.zeros((K3Z, K3Y, K3X))
    for oz in range(K3Z):
        for oy in range(K3Y):
            for ox in range(K3X):
                s = 0.0
                for t in range(27):
                    dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
                    r = ((oz + 1 + dz) * K3HY + (oy + 1 + dy)) * K3HX + (ox + 1 + dx)
                    assert 0 <= r < rows
                    s += D[r, t]
                got[oz, oy, ox] = s
    want = np.zeros((K3Z, K3Y, K3X))
    for t in range(27):
        dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
        sl = (slice(1 + dz, 1 + dz + K3Z), slice(1 + dy, 1 + dy + K3Y), slice(1 + dx, 1 + dx + K3X))
        want += 0.5 * (pos[sl] @ w[t] - neg[sl] @ w[t])
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12)


def k1_off(r, c8):
    """Byte offset of im2col row r, 8-element K chunk c8 (k_layer1_tc)."""
    return (r >> 3) * 512 + c8 * 128 + (r & 7) * 16


def test_layer1_im2col_layout_tiles_its_plane():
    """128 rows x 4 K chunks of 16 bytes fill one 8 KB plane exactly once; the
    MMA's K halves start 256 B apart with LBO 128 and SBO 512; the 16 x 32
    weight operand ends at 1 KB."""
    offs = sorted(k1_off(r, c) for r in range(128) for c in range(4))
    assert offs == list(range(0, 8192, 16))
    for r in range(128):
        for c in range(4):
            kh, cc = divmod(c, 2)
            assert k1_off(r, c) == kh * 256 + (r >> 3) * 512 + cc * 128 + (r & 7) * 16
    assert max(k1_off(co, t >> 3) + (t & 7) * 2 for co in range(16) for t in range(32)) == 1022


def test_layer1_im2col_product_equals_the_conv():
    """Each row = the 27 neighbours of its point (5 zero taps); the K = 32
    product with w1[t][0][co] gives layer 1's 16 pre-activations."""
    rng = np.random.default_rng(4)
    hz, hy, hx = 6, 10, 18
    field = rng.standard_normal((hz, hy, hx))
    w = rng.standard_normal((27, CH))
    Bw = np.zeros((32, CH))
    Bw[:27] = w
    for q in range(4):
        A = np.zeros((128, 32))
        for m in range(128):
            mx, my = m % 16, m // 16
            for t in range(27):
                dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
                A[m, t] = field[q + 1 + dz, my + 1 + dy, mx + 1 + dx]
        got = (A @ Bw).reshape(8, 16, CH)
        want = np.zeros((8, 16, CH))
        for t in range(27):
            dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
            want += field[q + 1 + dz, 1 + dy:9 + dy, 1 + dx:17 + dx][..., None] * w[t]
        assert np.allclose(got, want, rtol=1e-12, atol=1e-12)
