"""Shared helpers of the GPU parity tests (imported by tests only)."""
import numpy as np
import torch

from oracle import lbm_oracle as O

FACE_NAMES = ("input", "output", "back", "forward", "bottom", "top")
CODE_NAME = {11000: "PERIODICAL", 1200: "WALL", 1201: "WALL_WITH_SPEED", 1400: "NON_EQUILIBRIUM"}


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("GPU test without a CUDA device")
    from funlbm_b200 import _lib, build

    build.build()
    _lib.load()


def boundary_json(codes, uw=None):
    out = {}
    for i, k in enumerate(FACE_NAMES):
        out[k] = {"code": CODE_NAME[int(codes[i])]}
        if uw is not None and int(codes[i]) == 1201:
            out[k]["uw"] = [float(v) for v in uw[i]]
    return out


def smooth_f0(q, shape, amp, seed, rho_amp=0.01):
    """A smooth, non-equilibrium-free initial field (feq of a random smooth
    velocity) as float32 [X, Y, Z, Q]."""
    e, w, _ = O.velocity_set(q)
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
    rho = 1 + rho_amp * np.sin(2 * np.pi * (xs / X + ys / Y + zs / Z) + ph[0])
    eu = u @ e.T * 3.0
    feq = rho[..., None] * w * (1 + eu + eu * eu / 2 - 1.5 * (u * u).sum(-1, keepdims=True))
    return feq.astype(np.float32)


def to_np(t):
    return t.detach().float().cpu().numpy()


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def lbm_config(q, size, mu, codes, uw=None, body_force=None, storage="fp32", particles=(),
               gl=0.0, fused=True, ibm_mode="reference"):
    from funlbm_b200.lbm import Config

    flow = {"size": list(size), "param_type": "D3Q%d" % q, "param": {"mu": mu, "gl": gl},
            "boundary": boundary_json(codes, uw), "precision": {"storage": storage}}
    if body_force is not None:
        flow["body_force"] = list(body_force)
    return Config().from_json({"device": "cuda", "dt": 1, "dx": 1, "flow": flow,
                               "particles": list(particles), "fused": fused,
                               "log_per_steps": 10 ** 9, "file": {"per_steps": 10 ** 9},
                               "ibm": {"mode": ibm_mode}})


def init_with(lbm, f0):
    """The golden fixtures' initialisation: FlowD3.init, replace f, refresh the
    moments, LBMD3._init's collision, particle init."""
    lbm.flow.init()
    if f0 is not None:
        lbm.flow.f = torch.tensor(f0, device="cuda")
        lbm.flow.update_u_rou()
    lbm.flow.cul_equ()
    lbm.particle_swarm.init()


def run(lbm, n):
    for _ in range(n):
        lbm.run_step(step=lbm.step)
        lbm.step += 1
