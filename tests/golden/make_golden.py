"""Generate golden vectors by running the reference funlbm 1.2.0 itself.

Run in the build container (where the reference source is mounted):

    python tests/golden/make_golden.py --reference <funlbm checkout>/src

(or set FUNLBM_REFERENCE_SRC instead of --reference).

The reference imports five packages that are absent here (funutil, funtable,
funvtk, funtecplot, h5py); ``tests/golden/_stubs`` holds project-written
stand-ins for them (pass-through decorators, a ``deep_get`` dict lookup, no-op
loggers and writers).  Two reference paths crash as shipped and are patched
minimally before they are recorded (the same fixes the oracle assumes):

* WALL_WITH_SPEED: ``Boundary.get("uw")`` returns the wall velocity as a
  float32 tensor instead of failing inside ``x or default``;
* NON_EQUILIBRIUM: the inlet ``u_max`` reaches ``init_u`` as a Python float
  instead of a tensor.

Outputs (small float32 ``.npz`` files next to this script):

* ``kat_q{13,15,19,27}.npz``: one call each of ``cul_equ``, ``f_stream``,
  ``update_u_rou`` and ``cul_equ2`` on random states and random face mixes;
* ``steps_q{13,15,19,27}.npz``: ``LBMD3.run_step`` sequences without particles;
* ``particles.npz``: ``LBMD3.run_step`` sequences with a sphere and an
  ellipsoid, per-step particle state and flow moments;
* ``markers.npz``: reference marker sets for the sphere / ellipsoid shapes used
  by the benchmark configurations.

Nothing here runs at test time; the tests only read the ``.npz`` files.
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

FACES = ("input", "output", "back", "forward", "bottom", "top")
CODES = {"PERIODICAL": 11000, "WALL": 1200, "WALL_WITH_SPEED": 1201, "NON_EQUILIBRIUM": 1400}


def _setup(ref_src):
    sys.path.insert(0, os.path.join(HERE, "_stubs"))
    sys.path.insert(0, ref_src)
    import torch  # noqa: F401

    import funlbm.flow.d3.base as d3base

    orig = d3base.init_u

    def init_u_fixed(a, b, u_max=0.01, n_max=100):
        return orig(a, b, u_max=float(u_max), n_max=n_max)

    d3base.init_u = init_u_fixed


def _patch_uw(flow, face_uw):
    import torch

    for face, uw in face_uw.items():
        b = getattr(flow.config.boundary, face)
        t = torch.tensor(uw, dtype=torch.float32)
        b.get = (lambda tt: (lambda key, default=None: tt if key == "uw" else None))(t)


def _flow(q, size, mu, faces, face_uw=None, Re=10.0):
    from funlbm.flow import FlowConfig, create_flow

    cfg = FlowConfig().from_json({
        "size": list(size), "param_type": "D3Q%d" % q,
        "param": {"mu": mu, "Re": Re},
        "boundary": {k: {"code": v} for k, v in faces.items()},
    })
    fl = create_flow(cfg, device="cpu")
    if face_uw:
        _patch_uw(fl, face_uw)
    return fl


def _rand_state(rng, q, shape, w):
    X, Y, Z = shape
    f = w[None, None, None, :] * (1 + 0.1 * rng.standard_normal((X, Y, Z, q)))
    u = 0.05 * rng.standard_normal((X, Y, Z, 3))
    rou = 1 + 0.02 * rng.standard_normal((X, Y, Z, 1))
    fol = 1e-3 * rng.standard_normal((X, Y, Z, 3))
    return [a.astype(np.float32) for a in (f, u, rou, fol)]


def _face_mix(rng, allow_neq):
    faces = {}
    for k in FACES:
        opts = ["PERIODICAL", "WALL", "WALL_WITH_SPEED"]
        if allow_neq and k in ("input", "output"):
            opts.append("NON_EQUILIBRIUM")
        faces[k] = opts[rng.integers(len(opts))]
    uw = {k: (0.02 * rng.standard_normal(3)).astype(np.float32).tolist()
          for k in FACES if faces[k] == "WALL_WITH_SPEED"}
    return faces, uw


def _pack_faces(faces, uw):
    codes = np.array([CODES[faces[k]] for k in FACES], np.int32)
    uwa = np.zeros((6, 3), np.float32)
    for i, k in enumerate(FACES):
        if k in uw:
            uwa[i] = uw[k]
    return codes, uwa


def make_kat(q, rng, ncase=4):
    import torch

    out = {}
    size = (4, 5, 6)
    for c in range(ncase):
        faces, uw = _face_mix(rng, allow_neq=(c % 2 == 1))
        fl = _flow(q, size, 0.1 + 0.05 * c, faces, uw, Re=10.0 + c)
        fl.init()
        w = fl.param.w.numpy()[0]
        f, u, rou, fol = _rand_state(rng, q, tuple(s + 1 for s in size), w)
        pre = "c%d_" % c
        codes, uwa = _pack_faces(faces, uw)
        out[pre + "faces"] = codes
        out[pre + "uw"] = uwa
        out[pre + "mu"] = np.float64(0.1 + 0.05 * c)
        out[pre + "Re"] = np.float64(10.0 + c)
        out[pre + "f"], out[pre + "u"], out[pre + "rou"], out[pre + "FOL"] = f, u, rou, fol
        # cul_equ
        fl.f, fl.u, fl.rou, fl.FOL = (torch.tensor(a) for a in (f, u, rou, fol))
        fl.cul_equ()
        out[pre + "collide_f"] = fl.f.numpy().copy()
        out[pre + "collide_feq"] = fl.feq.numpy().copy()
        # f_stream (feq from the collision above is live, as in a real step)
        fl.f = torch.tensor(f)
        fl.f_stream()
        out[pre + "stream_f"] = fl.f.numpy().copy()
        # update_u_rou on the streamed populations
        fl.FOL = torch.tensor(fol)
        fl.update_u_rou()
        out[pre + "moments_rou"] = fl.rou.numpy().copy()
        out[pre + "moments_u"] = fl.u.numpy().copy()
        out[pre + "moments_p"] = fl.p.numpy().copy()
        # cul_equ2 with the given u and FOL
        fl.f, fl.u, fl.FOL = torch.tensor(f), torch.tensor(u), torch.tensor(fol)
        fl.cul_equ2()
        out[pre + "force_f"] = fl.f.numpy().copy()
    out["ncase"] = np.int32(ncase)
    return out


def _lbm(q, size, mu, faces, particles=(), gl=0.0):
    from funlbm.lbm import LBMD3, Config

    cfg = Config().from_json({
        "device": "cpu", "dt": 1, "dx": 1,
        "flow": {"size": list(size), "param_type": "D3Q%d" % q,
                 "param": {"mu": mu, "gl": gl},
                 "boundary": {k: {"code": v} for k, v in faces.items()}},
        "particles": list(particles),
        "file": {"per_steps": 1000000},
    })
    return LBMD3(config=cfg)


def _smooth_f0(q, shape, w, e, amp, seed):
    rng = np.random.default_rng(seed)
    X, Y, Z = shape
    xs = np.arange(X)[:, None, None]
    ys = np.arange(Y)[None, :, None]
    zs = np.arange(Z)[None, None, :]
    ph = rng.uniform(0, 2 * np.pi, 3)
    ux = amp * np.sin(2 * np.pi * ys / Y + ph[0]) * np.cos(2 * np.pi * zs / Z)
    uy = amp * np.sin(2 * np.pi * zs / Z + ph[1]) * np.cos(2 * np.pi * xs / X)
    uz = amp * np.sin(2 * np.pi * xs / X + ph[2]) * np.cos(2 * np.pi * ys / Y)
    u = np.stack(np.broadcast_arrays(ux, uy, uz), -1)
    rho = 1 + 0.01 * np.sin(2 * np.pi * (xs / X + ys / Y + zs / Z) + ph[0])
    eu = u @ e.T * 3.0
    feq = rho[..., None] * w * (1 + eu + eu * eu / 2 - 1.5 * (u * u).sum(-1, keepdims=True))
    return feq.astype(np.float32)


def _init_with(lbm, f0):
    import torch

    lbm.flow.init()
    if f0 is not None:
        lbm.flow.f = torch.tensor(f0)
        lbm.flow.update_u_rou()
    lbm.flow.cul_equ()
    lbm.particle_swarm.init()


def make_steps(q, rng, ncase=4, nsteps=12):
    out = {}
    size = (6, 7, 8)
    for c in range(ncase):
        faces = {k: ("PERIODICAL" if rng.random() < 0.5 else "WALL") for k in FACES}
        mu = 0.05 + 0.05 * c
        lbm = _lbm(q, size, mu, faces)
        shape = tuple(s + 1 for s in size)
        f0 = _smooth_f0(q, shape, lbm.flow.param.w.numpy()[0], lbm.flow.param.e.numpy(), 0.04, 100 + c)
        _init_with(lbm, f0)
        for _ in range(nsteps):
            lbm.run_step(step=lbm.step)
            lbm.step += 1
        pre = "c%d_" % c
        out[pre + "faces"] = np.array([CODES[faces[k]] for k in FACES], np.int32)
        out[pre + "mu"] = np.float64(mu)
        out[pre + "f0"] = f0
        out[pre + "f"] = lbm.flow.f.numpy().copy()
        out[pre + "u"] = lbm.flow.u.numpy().copy()
        out[pre + "rou"] = lbm.flow.rou.numpy().copy()
    out["ncase"] = np.int32(ncase)
    out["nsteps"] = np.int32(nsteps)
    out["size"] = np.array(size, np.int32)
    return out


PARTICLE_CASES = [
    # (name, q, size, mu, gl, faces, particle configs, steps, f0 amplitude)
    ("sphere_mid", 19, (20, 16, 16), 0.1, 2e-3, "WALL",
     [{"type": "sphere", "r": 3, "rou": 1.5, "coord": {"center": [10, 8, 8]}}], 6, 0.03),
    ("ellipsoid_wall", 19, (18, 14, 14), 0.08, -1e-3, "WALL",
     [{"a": 4, "b": 3, "c": 2.5, "rou": 1.2, "coord": {"center": [3.2, 7.4, 6.6], "alpha": 0.3, "beta": 0.7, "gamma": -0.4}}], 5, 0.02),
    ("two_spheres_q27", 27, (16, 14, 18), 0.12, 1e-3, "PERIODICAL",
     [{"type": "sphere", "r": 2.5, "rou": 1.3, "coord": {"center": [6, 7, 6]}},
      {"type": "sphere", "r": 2.5, "rou": 0.8, "coord": {"center": [9, 7, 10.5]}}], 5, 0.03),
]


def make_particles():
    out = {}
    for name, q, size, mu, gl, face, parts, nsteps, amp in PARTICLE_CASES:
        faces = {k: face for k in FACES}
        lbm = _lbm(q, size, mu, faces, parts, gl=gl)
        shape = tuple(s + 1 for s in size)
        f0 = _smooth_f0(q, shape, lbm.flow.param.w.numpy()[0], lbm.flow.param.e.numpy(), amp, 7)
        _init_with(lbm, f0)
        pre = name + "_"
        out[pre + "f0"] = f0
        for i, p in enumerate(lbm.particle_swarm.particles):
            out[pre + "p%d_lagrange" % i] = p._lagrange.numpy().copy()
        hist = {k: [] for k in ("cx", "cu", "cw", "cF", "cT", "lx", "lF", "lu", "lrou", "angle")}
        flow_hist = {k: [] for k in ("rou", "u", "FOL")}
        for _ in range(nsteps):
            lbm.run_step(step=lbm.step)
            lbm.step += 1
            for k in hist:
                hist[k].append(np.stack([
                    (p.coord.angle if k == "angle" else getattr(p, k)).numpy().copy()
                    for p in lbm.particle_swarm.particles]) if k not in ("lx", "lF", "lu", "lrou")
                    else np.concatenate([getattr(p, k).numpy().copy() for p in lbm.particle_swarm.particles]))
            flow_hist["rou"].append(lbm.flow.rou.numpy().copy())
            flow_hist["u"].append(lbm.flow.u.numpy().copy())
            flow_hist["FOL"].append(lbm.flow.FOL.numpy().copy())
        for k, v in hist.items():
            out[pre + k] = np.stack(v)
        # full flow fields only for the last step (keeps fixtures small)
        out[pre + "rou_last"] = flow_hist["rou"][-1]
        out[pre + "u_last"] = flow_hist["u"][-1]
        out[pre + "FOL_last"] = flow_hist["FOL"][-1]
        # first-step FOL (markers at the origin) as well
        out[pre + "FOL_first"] = flow_hist["FOL"][0]
        out[pre + "rou_mean"] = np.array([r.mean() for r in flow_hist["rou"]], np.float64)
        out[pre + "masses"] = np.array([float(p.mass) for p in lbm.particle_swarm.particles])
        out[pre + "areas"] = np.array([float(p.area) for p in lbm.particle_swarm.particles])
        out[pre + "inertia"] = np.stack([p.I.numpy() for p in lbm.particle_swarm.particles])
    return out


def make_markers():
    from funlbm.particle import ParticleConfig, create_particle

    out = {}
    shapes = {
        "sphere_r8": {"type": "sphere", "r": 8, "coord": {"center": [0, 0, 0]}},
        "sphere_r4": {"type": "sphere", "r": 4, "coord": {"center": [0, 0, 0]}},
        "ellipsoid_644": {"a": 6, "b": 4, "c": 4, "coord": {"center": [0, 0, 0]}},
        "ellipsoid_1075": {"a": 10, "b": 7, "c": 5, "coord": {"center": [0, 0, 0]}},
    }
    for name, cfg in shapes.items():
        pc = ParticleConfig().from_json(cfg)
        p = create_particle(pc, device="cpu")
        p.init()
        out[name] = p._lagrange.numpy().copy()
        out[name + "_mass_area_I"] = np.concatenate([[float(p.mass), float(p.area)], p.I.numpy()])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("FUNLBM_REFERENCE_SRC"),
                    help="the funlbm source tree (its src/ directory)")
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    if not args.reference:
        ap.error("pass --reference or set FUNLBM_REFERENCE_SRC")
    _setup(args.reference)
    import torch

    torch.set_num_threads(4)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        try:
            rng = np.random.default_rng(20261203)
            for q in (13, 15, 19, 27):
                np.savez_compressed(os.path.join(args.out, "kat_q%d.npz" % q), **make_kat(q, rng))
            for q in (19, 27):
                np.savez_compressed(os.path.join(args.out, "steps_q%d.npz" % q), **make_steps(q, rng))
            np.savez_compressed(os.path.join(args.out, "particles.npz"), **make_particles())
            np.savez_compressed(os.path.join(args.out, "markers.npz"), **make_markers())
            # D3Q13 / D3Q15 step sequences, from a generator of their own (the
            # files above keep their random states)
            rng13 = np.random.default_rng(20261204)
            for q in (13, 15):
                np.savez_compressed(os.path.join(args.out, "steps_q%d.npz" % q), **make_steps(q, rng13))
        finally:
            os.chdir(cwd)


if __name__ == "__main__":
    main()
