"""The TMA-staged FP32 colour passes (kv_pass_tma: full sweep, zero-guess
forward and backward) against the 4-row kernels they replace on large levels.

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
