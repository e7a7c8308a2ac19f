"""The bounds-checked build (liblbm_b200_checked.so, -DLBM_BOUNDS_CHECK):
a battery of lattices and particle runs -- pitched rows of odd length in
every launch shape, WALL_WITH_SPEED faces, chunked force fields, FP16 and
FP64 storage, the fused particle chain with tiled spreading, the step
statistics and the reference call sequence -- runs in child processes once
on the checked library and once on the normal one.  The checked run must
count no index violation and give the normal run's results bit for bit --
except the step statistics' means, float64 sums that blocks add atomically
in no fixed order, which must agree to 1e-12 of the values' range (their minima and maxima bit
for bit)."""
import json
import os
import subprocess
import sys

import pytest

from tests.gpu_util import require_cuda

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import hashlib, itertools, json, os, sys
import numpy as np
root, checked = sys.argv[1], sys.argv[2] == "1"
sys.path.insert(0, root)
import torch
from funlbm_b200 import _lib, build
build.build(checked=checked)
lib = _lib.load()
assert lib._name.endswith("liblbm_b200_checked.so" if checked else "liblbm_b200.so"), lib._name
from funlbm_b200.lattice import Lattice, make_force, tau_float32
from funlbm_b200.lbm import LBMD3, Config
from funlbm_b200.tune import CANDIDATES, STORAGE_BITS, shape_ok
from tests.gpu_util import init_with, lbm_config, run, smooth_f0

out = {}
stats = {}
def h(t):
    return hashlib.sha256(t.detach().cpu().numpy().tobytes()).hexdigest()

rng = np.random.default_rng(5)
shape = (9, 8, 13)
n = shape[0] * shape[1] * shape[2]
nch = (n + 31) // 32
kind = rng.integers(0, 4, nch)
for storage in ("fp32", "fp16s", "fp64"):
    dt = torch.float64 if storage == "fp64" else torch.float32
    co = torch.tensor(((kind == 1) | (kind == 3)).astype(np.uint8), device="cuda")
    cn = torch.tensor(((kind == 2) | (kind == 3)).astype(np.uint8), device="cuda")
    fo = torch.tensor(1e-4 * rng.standard_normal(3 * n), device="cuda", dtype=dt)
    fn = torch.tensor(1e-4 * rng.standard_normal(3 * n), device="cuda", dtype=dt)
    force = make_force((0, 0, 0), (1e-6, 0, 0), fo, fn, co, cn)
    for q in (19, 27):
        f0 = smooth_f0(q, shape, 0.04, q)
        f0 = torch.tensor(np.ascontiguousarray(np.moveaxis(f0, -1, 0)), device="cuda", dtype=dt)
        bits = STORAGE_BITS[storage]
        for (nodes, threads), pitch, zf in itertools.product(
                CANDIDATES[bits], (False, True), ((1201, 1201), (1200, 11000))):
            lat = Lattice(q, shape, [1200, 11000, 11000, 1200, *zf], tau_float32(0.07),
                          storage=storage, face_uw=[(0.01, 0.0, -0.01)] * 6, device="cuda",
                          pitch=pitch)
            if not shape_ok(nodes, lat.pz, bits, shape[2]):
                continue
            lat.set_launch_shape(nodes, threads)
            lat.init(f0)
            for _ in range(3):
                lat.step(force)
            f = torch.empty(q * lat.n, device="cuda", dtype=dt)
            lat.observe(force, f=f)
            key = "%s_q%d_%d_%d_%d_%d" % (storage, q, nodes, threads, pitch, zf[0])
            out["lat_" + key] = h(f)
            stats["stats_" + key] = lat.stats(force).cpu().tolist()
parts = [{"type": "sphere", "r": 3, "rou": 1.4, "coord": {"center": [2.4, 8.0, 9.1]}},
         {"type": "ellipsoid", "a": 3, "b": 2, "c": 2.5, "rou": 0.7,
          "coord": {"center": [12.5, 11.3, 7.6], "alpha": 0.3, "beta": -0.5, "gamma": 0.2}}]
for storage in ("fp32", "fp64"):
    for fused in (True, False):
        if storage == "fp64" and not fused:
            continue
        lbm = LBMD3(config=lbm_config(19, (16, 16, 17), 0.1, [1200] * 6, particles=parts,
                                      gl=1e-3, storage=storage, fused=fused,
                                      body_force=[0, 1e-6, 0]))
        init_with(lbm, None)
        run(lbm, 12)
        p = lbm.particle_swarm.particles
        key = "lbm_%s_%s" % (storage, "fused" if fused else "ref")
        out[key] = [h(lbm.flow.rou), h(lbm.flow.u)] + [h(x.cx) for x in p]
        stats[key + "_stats"] = lbm.flow.step_stats().cpu().tolist()
torch.cuda.synchronize()
print(json.dumps({"faults": int(lib.lbm_debug_bounds_faults(0)), "hashes": out, "stats": stats}))
"""


def _child(checked):
    env = dict(os.environ, FUNLBM_B200_CHECKED="1" if checked else "0")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, "1" if checked else "0"],
                       capture_output=True, text=True, timeout=1200, env=env)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_checked_build_counts_no_violation_and_matches():
    require_cuda()
    normal = _child(False)
    checked = _child(True)
    assert normal["faults"] == -1
    assert checked["faults"] == 0
    assert len(checked["hashes"]) > 20
    assert checked["hashes"] == normal["hashes"]
    assert checked["stats"].keys() == normal["stats"].keys() and len(normal["stats"]) > 20
    for key, a in normal["stats"].items():
        b = checked["stats"][key]
        for k in range(9):
            if k % 3 == 1:     # mean: float64 atomics in no fixed order
                scale = abs(a[k - 1]) + abs(a[k + 1])   # the values' range
                assert abs(a[k] - b[k]) <= 1e-12 * scale, (key, k)
            else:
                assert a[k] == b[k], (key, k)
