"""The CG step as two kernels (HPCGB200_CG_STEP=2): a persistent cooperative
kernel for r.z, beta, the p update and the SpMV with p.Ap and alpha (two
bounded grid barriers), then one for the r/x update, ||r|| and the loop
control (src/CG.cpp:148-184).  Its scalars come from other (fixed) reduction
partitions than the five-kernel body's, so the residual history must agree
to summation-order rounding, with the same iteration count, in the FP64 and
the mixed modes; the kernels per iteration drop by three."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import rochpcg_b200 as R

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import rochpcg_b200 as R
from rochpcg_b200.rhs import normal_rhs
dims = tuple(json.loads(sys.argv[2])); mode = int(sys.argv[3])
P = R.Problem(*dims)
P.set_rhs(normal_rhs(P.rows[0], 3))
r = P.cg(500, 1e-9, mode=mode)
print(json.dumps({"hist": r["hist"].tolist(), "niters": r["niters"], "kpi": P.kernels_per_iteration(mode),
                  "true": P.true_residual()}))
"""


def run(dims, mode, step):
    env = dict(os.environ, HPCGB200_CG_STEP=str(step))
    res = subprocess.run([sys.executable, "-c", CHILD, ROOT, json.dumps(list(dims)), str(mode)], env=env,
                         capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    return json.loads(res.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("dims", [(32, 32, 32), (24, 40, 56), (64, 64, 64)])
@pytest.mark.parametrize("mode_name", ["MODE_FP64", "MODE_MIXED"])
def test_two_kernel_step_matches_five_kernel_body(dims, mode_name):
    mode = getattr(R, mode_name)
    five, two = run(dims, mode, 5), run(dims, mode, 2)
    assert abs(two["niters"] - five["niters"]) <= 1
    k = min(len(two["hist"]), len(five["hist"]))
    h5, h2 = np.array(five["hist"][:k]), np.array(two["hist"][:k])
    live = h5 / h5[0] > 1e-11
    # FP64: only the dot products' summation order differs (1e-6 over the
    # solve, as against the CPU restatement); mixed: the FP32 V-cycle turns
    # last-bit differences of r into FP32 rounding differences of z, which
    # compound to about 1e-6 by 1e-9 -- 1e-4 bounds them
    rtol = 1e-6 if mode == R.MODE_FP64 else 1e-4
    assert np.allclose(h2[live], h5[live], rtol=rtol, atol=0)
    assert two["true"] <= 2e-9
    assert five["kpi"] - two["kpi"] == 3
