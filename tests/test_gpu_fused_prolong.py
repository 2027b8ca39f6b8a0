"""The prolongation carried by the coarse level's final smoother passes
(xf[pro_f[row]] += x_new in the pass that finalizes each coarse row) must give
the bits of the separate ComputeProlongation launch after the coarse solve
(src/ComputeMG.cpp:86-90, src/ComputeProlongation.cpp:39-59), in the FP64,
FP64-stencil and FP32 V-cycles, and remove one launch per coarse level.  The
fused form runs in a child process with HPCGB200_FUSED_PROLONG=1 (the default
is the separate launch, measured faster)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import rochpcg_b200 as R
from gpu_util import host, sync, to_dev

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import rochpcg_b200 as R
dims = tuple(json.loads(sys.argv[2])); mode = int(sys.argv[3]); out = sys.argv[4]
P = R.Problem(*dims)
r = np.random.default_rng(7).normal(size=P.rows[0])
rd = torch.from_numpy(r).cuda(); zd = torch.empty_like(rd)
torch.cuda.synchronize()
P.mg(rd.data_ptr(), zd.data_ptr(), mode=mode)
torch.cuda.ExternalStream(P.stream_handle).synchronize(); torch.cuda.synchronize()
np.save(out, zd.cpu().numpy())
print(json.dumps({"kpi": P.kernels_per_iteration(mode)}))
"""


@pytest.mark.parametrize("dims", [(32, 32, 32), (24, 40, 56)])
@pytest.mark.parametrize("mode_name", ["MODE_FP64", "MODE_FP64_STENCIL", "MODE_MIXED"])
def test_fused_prolongation_bitwise_equal_to_separate(dims, mode_name, tmp_path):
    """In-process: the default (separate launch); child: the fused form."""
    mode = getattr(R, mode_name)
    P = R.Problem(*dims)
    r = np.random.default_rng(7).normal(size=P.rows[0])
    rd, zd = to_dev(r), torch.empty(P.rows[0], dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    P.mg(rd.data_ptr(), zd.data_ptr(), mode=mode)
    sync(P)
    separate = host(zd)
    kpi_separate = P.kernels_per_iteration(mode)
    P.close()
    out = str(tmp_path / "z.npy")
    env = dict(os.environ, HPCGB200_FUSED_PROLONG="1")
    res = subprocess.run([sys.executable, "-c", CHILD, ROOT, json.dumps(list(dims)), str(mode), out], env=env,
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    fused = np.load(out)
    assert np.array_equal(fused, separate)
    kpi_fused = json.loads(res.stdout.strip().splitlines()[-1])["kpi"]
    assert kpi_separate - kpi_fused == 3  # one prolongation launch per coarse level
