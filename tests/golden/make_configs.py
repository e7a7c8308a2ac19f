"""Generate the long-horizon fixtures of the benchmark configurations by
running the reference funlbm 1.2.0 itself on the CPU.

    python tests/golden/make_configs.py --reference <funlbm checkout>/src [--only config1|config2]
                                        [--device cuda]

(or set FUNLBM_REFERENCE_SRC instead of --reference).  Like ``make_golden.py``
it puts the project-written stand-ins of ``tests/golden/_stubs`` in front of
the reference for its five absent helper packages.

* ``config1_poiseuille.npz`` -- the Poiseuille channel: D3Q19, size
  [32, 32, 64] (33 x 33 x 65 nodes), mu = 0.1 (tau = 0.8), WALL on the x and y
  faces, PERIODICAL on the z faces, uniform body force (0, 0, 1e-6), rho = 1,
  u = 0, 2000 steps.  The reference has no body-force option; the script adds
  the force to FOL right after ``lagrange_to_flow`` (lbm/lbm3d.py:102-119)
  resets it, which is where this build's ``flow.body_force`` extension and
  the oracle apply it.  Recorded: rho and u after steps 1000 and 2000.  The
  same file carries the float64 run of the oracle (``oracle/lbm_oracle.py``)
  of this configuration -- rho and u on the mid plane z = 32 and the mean
  density after steps 1000 and 2000 -- the yardstick of float32 rounding: the
  reference's float32 run drifts from it by ~2.5e-5 in rho (its total mass
  grows) and ~1.4e-2 of max|u| in u over 2000 steps.
* ``config2_sphere.npz`` -- the single-sphere free fall in the reference's
  axes (gravity acts along +x scaled by 1 - rho_p / rho_f, so the fall is
  along -x): D3Q19, size [160, 64, 64] (161 x 65 x 65 nodes), every face
  WALL, mu = 0.0666667 (tau = 0.7), a sphere of radius 8 (1160 markers) at
  (130, 32, 32) with density 1.5, gl = 2e-5, 5000 steps.  Recorded: the
  particle's cx, cu, cw, cF and rotation vector after every step, and rho /
  u on the mid plane z = 32 at the end.

CPU time: a few minutes for config 1 and one to several hours for config 2
(the reference's interpolation and spreading are Python loops over the
markers).  ``--device cuda`` runs the reference's own torch code with its
flow and particles on the GPU instead (created by its ``create_flow`` /
``create_particle_swarm`` and handed to ``LBMD3``, which otherwise always
builds them on the CPU: lbm/base.py:56-76, base/work.py:41-43); the
installed copy in baseline/_ref serves as ``--reference`` where the source
tree is not mounted.  The device is recorded in the fixture.
Nothing here runs at test time; the tests only read the ``.npz`` files.
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FACES = ("input", "output", "back", "forward", "bottom", "top")

CONFIG1 = {"size": (32, 32, 64), "mu": 0.1, "faces": ("WALL", "WALL", "WALL", "WALL",
                                                      "PERIODICAL", "PERIODICAL"),
           "body_force": (0.0, 0.0, 1e-6), "steps": 2000, "record": (1000, 2000)}
CONFIG2 = {"size": (160, 64, 64), "mu": 0.0666667, "gl": 2e-5, "steps": 5000,
           "particle": {"type": "sphere", "r": 8, "rou": 1.5, "coord": {"center": [130, 32, 32]}}}


def _setup(ref_src):
    sys.path.insert(0, os.path.join(HERE, "_stubs"))
    sys.path.insert(0, ref_src)


def _lbm(q, size, mu, faces, particles=(), gl=0.0, device="cpu"):
    from funlbm.flow import create_flow
    from funlbm.lbm import LBMD3, Config
    from funlbm.particle import create_particle_swarm

    cfg = Config().from_json({
        "device": device, "dt": 1, "dx": 1,
        "flow": {"size": list(size), "param_type": "D3Q%d" % q, "param": {"mu": mu, "gl": gl},
                 "boundary": {k: {"code": v} for k, v in zip(FACES, faces)}},
        "particles": list(particles), "file": {"per_steps": 10 ** 9},
    })
    if device == "cpu":
        return LBMD3(config=cfg)
    return LBMD3(config=cfg, flow=create_flow(cfg.flow_config, device=device),
                 particle_swarm=create_particle_swarm(cfg.particles, device=device), device=device)


def make_config1():
    import torch

    c = CONFIG1
    lbm = _lbm(19, c["size"], c["mu"], c["faces"])
    g = torch.tensor(c["body_force"], dtype=torch.float32)
    plain = lbm.lagrange_to_flow

    def lagrange_to_flow_with_force(*args, **kwargs):
        plain(*args, **kwargs)
        lbm.flow.FOL = lbm.flow.FOL + g

    lbm.lagrange_to_flow = lagrange_to_flow_with_force
    lbm.init()
    out = {"size": np.array(c["size"], np.int32), "mu": np.float64(c["mu"]),
           "body_force": np.array(c["body_force"], np.float64), "steps": np.int32(c["steps"])}
    t0 = time.time()
    for _ in range(c["steps"]):
        lbm.run_step(step=lbm.step)
        if lbm.step in c["record"]:
            out["rou_%d" % lbm.step] = lbm.flow.rou.numpy().copy()
            out["u_%d" % lbm.step] = lbm.flow.u.numpy().copy()
        lbm.step += 1
    print("config1: %d steps in %.1f s" % (c["steps"], time.time() - t0), flush=True)
    return out


def make_config1_oracle64():
    """The float64 oracle run of config 1 (mid-plane rho / u, mean rho)."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle import lbm_oracle as O

    c = CONFIG1
    code = {"WALL": O.WALL, "PERIODICAL": O.PERIODICAL}
    fl = O.OracleFlow(19, c["size"], c["mu"], dict(zip(O.FACES, [code[v] for v in c["faces"]])),
                      dtype=np.float64)
    lbm = O.OracleLBM(fl, body_force=c["body_force"])
    lbm.init(None)
    out = {}
    zmid = c["size"][2] // 2
    t0 = time.time()
    for s in range(1, c["steps"] + 1):
        lbm.run_step()
        lbm.step += 1
        if s in c["record"]:
            out["oracle64_rou_mid_%d" % s] = fl.rou[:, :, zmid].copy()
            out["oracle64_u_mid_%d" % s] = fl.u[:, :, zmid].copy()
            out["oracle64_rou_mean_%d" % s] = np.float64(fl.rou.mean())
    print("config1 oracle float64: %d steps in %.1f s" % (c["steps"], time.time() - t0), flush=True)
    return out


def make_config2(steps=None, device="cpu"):
    c = CONFIG2
    steps = c["steps"] if steps is None else steps
    lbm = _lbm(19, c["size"], c["mu"], ("WALL",) * 6, [c["particle"]], gl=c["gl"], device=device)
    lbm.init()
    p = lbm.particle_swarm.particles[0]
    hist = {k: [] for k in ("cx", "cu", "cw", "cF", "angle")}
    t0 = time.time()
    for s in range(steps):
        lbm.run_step(step=lbm.step)
        for k in hist:
            hist[k].append((p.coord.angle if k == "angle" else getattr(p, k)).cpu().numpy().copy())
        if not lbm.run_status:
            raise RuntimeError("the reference stopped its run at step %d" % lbm.step)
        lbm.step += 1
        if (s + 1) % 100 == 0:
            print("config2: step %d, %.1f s, cx %s" % (s + 1, time.time() - t0, hist["cx"][-1]),
                  flush=True)
    out = {k: np.stack(v).astype(np.float32) for k, v in hist.items()}
    zmid = c["size"][2] // 2
    out["rou_mid"] = lbm.flow.rou[:, :, zmid].cpu().numpy().copy()
    out["u_mid"] = lbm.flow.u[:, :, zmid].cpu().numpy().copy()
    out["lagrange"] = p._lagrange.cpu().numpy().copy()
    out["steps"] = np.int32(steps)
    out["device"] = np.array(str(device))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("FUNLBM_REFERENCE_SRC"),
                    help="the funlbm source tree (its src/ directory)")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", choices=["config1", "config2"], default=None)
    ap.add_argument("--config2-steps", type=int, default=None)
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--device", default="cpu", help="config 2 only: cpu or cuda")
    args = ap.parse_args()
    if not args.reference:
        ap.error("pass --reference or set FUNLBM_REFERENCE_SRC")
    _setup(args.reference)
    import torch

    torch.set_num_threads(args.threads)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            if args.only in (None, "config1"):
                out = make_config1()
                out.update(make_config1_oracle64())
                np.savez_compressed(os.path.join(args.out, "config1_poiseuille.npz"), **out)
            if args.only in (None, "config2"):
                np.savez_compressed(os.path.join(args.out, "config2_sphere.npz"),
                                    **make_config2(args.config2_steps, args.device))
        finally:
            os.chdir(cwd)


if __name__ == "__main__":
    main()
