"""The TMA-staged colour passes (kv_pass_tma: full sweep, zero-guess forward
and backward) against the 4-row kernels they replace on large levels, and the
separable product with TMA-staged planes (k64_spmv_sep) against its
eight-byte-copy staging.

The same V-cycle is run in this process (staged passes, the default) and in a
child process with HPCGB200_SWEEP_TMA=0 (4-row kernels everywhere); the
results must be equal bit for bit.  160^3 has 80-wide colour bricks on level
0, so its tiles run past the brick in x (zero-filled boxes, rows skipped);
256^3 stages levels 0 and 1.  The 4-row kernels are themselves pinned to the
FP32 restatement (tests/test_gpu_mixed.py, tests/test_gpu_parity_scale.py).
"""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, {root!r})
import rochpcg_b200 as R
P = R.Problem({n})
r = np.random.default_rng({seed}).normal(size=P.rows[0])
rd = torch.from_numpy(r).cuda()
zd = torch.empty_like(rd)
torch.cuda.synchronize()
P.mg(rd.data_ptr(), zd.data_ptr(), mode=R.MODE_MIXED)
torch.cuda.synchronize()
np.save({out!r}, zd.cpu().numpy())
P.close()
"""


def _vcycle_here(n, seed):
    import rochpcg_b200 as R

    P = R.Problem(n)
    try:
        r = np.random.default_rng(seed).normal(size=P.rows[0])
        rd = torch.from_numpy(r).cuda()
        zd = torch.empty_like(rd)
        torch.cuda.synchronize()
        P.mg(rd.data_ptr(), zd.data_ptr(), mode=R.MODE_MIXED)
        torch.cuda.synchronize()
        return zd.cpu().numpy()
    finally:
        P.close()


@pytest.mark.parametrize("n", [160, 256])
def test_staged_passes_equal_four_row_kernels(n, tmp_path):
    assert os.environ.get("HPCGB200_SWEEP_TMA", "1") != "0", "this process must run the staged passes"
    seed = 1000 + n
    out = str(tmp_path / "z.npy")
    env = dict(os.environ, HPCGB200_SWEEP_TMA="0")
    subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, n=n, seed=seed, out=out)], env=env, check=True,
                   timeout=600)
    want = np.load(out)
    got = _vcycle_here(n, seed)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


SEP_CHILD = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, {root!r})
import rochpcg_b200 as R
P = R.Problem(*{dims!r}, nlevels={nl})
x = torch.from_numpy(np.random.default_rng({seed}).normal(size=P.rows[0])).cuda()
y = torch.empty_like(x)
torch.cuda.synchronize()
P.spmv_mixed(0, x.data_ptr(), y.data_ptr())
torch.cuda.synchronize()
np.save({out!r}, y.cpu().numpy())
P.close()
"""


@pytest.mark.parametrize("dims,nl", [((320, 320, 320), 4), ((136, 90, 72), 1)])
def test_tma_staged_separable_product_equals_copy_staging(dims, nl, tmp_path):
    """The mixed CG's outer product with its planes staged by four TMA boxes
    each equals the eight-byte-copy staging (HPCGB200_SEP_TMA=0, child
    process) bit for bit: the same values land in shared memory and are summed
    in the same order.  136 x 90 x 72 (one level: 90 is not a multiple of 8)
    has tiles that run past the grid in x (64-wide tiles) and y (4-line
    tiles) and a last z chunk of 8 planes."""
    import rochpcg_b200 as R

    assert os.environ.get("HPCGB200_SEP_TMA", "1") != "0", "this process must stage by TMA"
    seed = 7 + dims[2]
    out = str(tmp_path / "y.npy")
    env = dict(os.environ, HPCGB200_SEP_TMA="0")
    subprocess.run([sys.executable, "-c", SEP_CHILD.format(root=ROOT, dims=dims, nl=nl, seed=seed, out=out)], env=env,
                   check=True, timeout=600)
    want = np.load(out)
    P = R.Problem(*dims, nlevels=nl)
    try:
        x = torch.from_numpy(np.random.default_rng(seed).normal(size=P.rows[0])).cuda()
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        P.spmv_mixed(0, x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(y.cpu().numpy().view(np.uint64), want.view(np.uint64))
    finally:
        P.close()
