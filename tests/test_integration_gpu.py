"""The second drop-in route: funlbm's own driver (the unmodified reference
installed in baseline/_ref) with a funlbm_b200 flow injected through
``LBMBase(flow=...)`` (lbm/base.py:56-76).  funlbm's ``LBMD3.run_step`` then
calls ``cul_equ`` / ``f_stream`` / ``update_u_rou`` / ``cul_equ2`` on the GPU
flow, one kernel each, and clears ``flow.FOL`` in place in
``lagrange_to_flow``; the result must match the run_step sequences the
reference recorded on its own CPU flow (tests/golden/steps_q*.npz) within the
tolerances of test_flow_gpu.py (f, rho 1e-5 relative; u 1e-5 of max|u|).

funlbm needs five helper packages that are not installable here; the
project-written stand-ins in tests/golden/_stubs replace them.  The run is a
child process so that those stand-ins (an ``h5py`` among them) never enter
the test process.  Particles stay on funlbm's CPU in this route (LBMBase
builds its swarm on Worker's default device), so the cases are
particle-free.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from tests.gpu_util import require_cuda

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "baseline", "_ref")
STUBS = os.path.join(ROOT, "tests", "golden", "_stubs")

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not os.path.isfile(os.path.join(REF, "funlbm", "__init__.py")),
                       reason="the reference is not installed in baseline/_ref"),
]

CHILD = r"""
import json, os, sys, tempfile
import numpy as np
root, ref, stubs, q, out = sys.argv[1:6]
sys.path[:0] = [stubs, ref, root]
import torch
from funlbm.lbm import LBMD3, Config
from funlbm_b200.flow import FlowConfig, create_flow
faces_names = ("input", "output", "back", "forward", "bottom", "top")
names = {11000: "PERIODICAL", 1200: "WALL"}
g = np.load(os.path.join(root, "tests", "golden", "steps_q%s.npz" % q))
res = {}
os.chdir(tempfile.mkdtemp())
for c in range(int(g["ncase"])):
    p = "c%d_" % c
    flow_json = {"size": [int(v) for v in g["size"]], "param_type": "D3Q%s" % q,
                 "param": {"mu": float(g[p + "mu"])},
                 "boundary": {k: {"code": names[int(v)]} for k, v in zip(faces_names, g[p + "faces"])}}
    cfg = Config().from_json({"dt": 1, "dx": 1, "flow": flow_json, "file": {"per_steps": 10 ** 9}})
    flow = create_flow(FlowConfig().from_json(flow_json), device="cuda")
    lbm = LBMD3(config=cfg, flow=flow)
    assert type(lbm).__module__.startswith("funlbm.")
    lbm.flow.init()
    lbm.flow.f = torch.tensor(g[p + "f0"], device="cuda")
    lbm.flow.update_u_rou()
    lbm.flow.cul_equ()
    lbm.particle_swarm.init()
    for _ in range(int(g["nsteps"])):
        lbm.run_step(step=lbm.step)
        lbm.step += 1
    np.savez(os.path.join(out, "c%d.npz" % c), f=lbm.flow.f.cpu().numpy(),
             u=lbm.flow.u.cpu().numpy(), rou=lbm.flow.rou.cpu().numpy())
    res[c] = True
print(json.dumps(res))
"""


@pytest.mark.parametrize("q", [13, 15, 19, 27])
def test_reference_driver_with_gpu_flow(q, tmp_path):
    require_cuda()
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, REF, STUBS, str(q), str(tmp_path)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    g = np.load(os.path.join(ROOT, "tests", "golden", "steps_q%d.npz" % q))
    for c in range(int(g["ncase"])):
        got = np.load(os.path.join(tmp_path, "c%d.npz" % c))
        p = "c%d_" % c
        for k in ("f", "rou"):
            ref = g[p + k]
            assert np.abs(got[k] - ref).max() <= 1e-5 * np.abs(ref).max(), (c, k)
        ref_u = g[p + "u"]
        assert np.abs(got["u"] - ref_u).max() <= 1e-5 * np.abs(ref_u).max() + 2e-7, c
