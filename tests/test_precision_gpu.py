"""GPU checks of the FP64 storage (the comparison run of the precision
figures) and of the 16-bit shifted storages against it.

* FP64 storage against the float64 oracle: every velocity set, random
  PERIODICAL / WALL / WALL_WITH_SPEED faces, a body force, ragged shapes, and
  a sedimenting sphere -- the same algorithm, so the two float64 codes agree
  to rounding (max relative error <= 1e-11 in f, rho and u after 25 steps;
  particle position / velocity within 1e-10 lattice units after 60 steps).
* FP32, FP16 and BF16 shifted storage against that FP64 run on a walled,
  forced, particle-laden case (D3Q19 and D3Q27): rho relative and u
  normalised by max|u| within 1e-3 for fp16s and 2e-2 for bf16s (the bounds
  of the periodic Taylor-Green case), particle position and velocity within
  1e-4 lattice units for fp32 and fp16s.

The uniform forces and gravity reach the kernels as float32, so the oracle is
given the float32-rounded values; its relaxation time is the float32 one the
lattice descriptor carries.
"""
import numpy as np
import pytest
import torch

from oracle import lbm_oracle as O
from tests.gpu_util import init_with, lbm_config, require_cuda, run, smooth_f0

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    require_cuda()


def to64(t):
    return t.detach().double().cpu().numpy()


def f32(v):
    return float(np.float32(v))


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("q", [13, 15, 19, 27])
def test_fp64_fused_vs_oracle64(q):
    """The fused step in FP64 storage equals the float64 oracle to rounding,
    with one and two nodes per thread (bit-identical to each other)."""
    from funlbm_b200.lbm import LBMD3

    rng = np.random.default_rng(300 + q)
    for case in range(2):
        size = tuple(int(v) for v in rng.integers(5, 12, 3))
        size = (size[0], size[1], size[2] | 1)          # even node count per row: vectors apply
        shape = tuple(s + 1 for s in size)
        codes = [int(c) for c in rng.choice([11000, 1200, 1201], 6)]
        uw = (0.02 * rng.standard_normal((6, 3))).astype(np.float32)
        bf = [f32(v) for v in 1e-5 * rng.standard_normal(3)]
        mu = float(rng.uniform(0.03, 0.2))
        f0 = smooth_f0(q, shape, 0.04, 40 * q + case)
        outs = []
        for nodes in (1, 2):
            lbm = LBMD3(config=lbm_config(q, size, mu, codes, uw, body_force=bf, storage="fp64"))
            init_with(lbm, f0)
            lbm.flow.lattice.set_launch_shape(nodes, 128 if nodes == 2 else 256)
            run(lbm, 25)
            assert lbm.check_status() == 0
            outs.append((to64(lbm.flow.f), to64(lbm.flow.u), to64(lbm.flow.rou)))
        for a, b in zip(*outs):
            assert np.array_equal(a, b)
        tau = float(np.float32(3 * mu + 0.5))
        faces = dict(zip(O.FACES, codes))
        fl = O.OracleFlow(q, size, mu, faces, {k: uw[i] for i, k in enumerate(O.FACES)},
                          dtype=np.float64, tau=tau)
        ref = O.OracleLBM(fl, body_force=bf)
        ref.init(f0.astype(np.float64))
        ref.run(25)
        f, u, rou = outs[0]
        assert rel(f, fl.f) <= 1e-11
        assert rel(rou, fl.rou) <= 1e-11
        assert np.abs(u - fl.u).max() <= 1e-11 * np.abs(fl.u).max()


def test_fp64_particles_vs_oracle64():
    """A sphere sedimenting in a closed box, 60 steps, FP64 storage and
    float64 particle state against the float64 oracle."""
    from funlbm_b200.lbm import LBMD3

    size, mu, gl = (40, 24, 24), 1.0 / 15, 2e-4
    parts = [{"type": "sphere", "r": 4, "rou": 1.5, "coord": {"center": [28, 12, 12]}}]
    lbm = LBMD3(config=lbm_config(19, size, mu, [1200] * 6, particles=parts, gl=gl,
                                  storage="fp64"))
    init_with(lbm, None)
    run(lbm, 60)
    assert lbm.check_status() == 0
    p = lbm.particle_swarm.particles[0]
    assert p.cx.dtype == torch.float64
    fl = O.OracleFlow(19, size, mu, dict(zip(O.FACES, [1200] * 6)), dtype=np.float64,
                      tau=float(np.float32(3 * mu + 0.5)))
    op = O.OracleParticle(to64(p._lagrange), float(p.mass), float(p.area), to64(p.I), 1.5,
                          [28, 12, 12], [np.pi / 2, 0, 0], dtype=np.float64)
    ref = O.OracleLBM(fl, [op], gl=f32(gl))
    ref.init(None)
    ref.run(60)
    assert np.abs(op.cx - 28).max() > 1e-3                 # it moved
    for k in ("cx", "cu", "cw"):
        assert np.abs(to64(getattr(p, k)) - getattr(op, k)).max() <= 1e-10, k
    assert rel(to64(lbm.flow.rou), fl.rou) <= 1e-11
    assert np.abs(to64(lbm.flow.u) - fl.u).max() <= 1e-9 * np.abs(fl.u).max()


def _sphere_run(q, storage, steps):
    from funlbm_b200.lbm import LBMD3

    size = (30, 22, 25)
    codes = [1200, 1200, 11000, 11000, 1200, 1200]
    parts = [{"type": "sphere", "r": 4, "rou": 1.3, "coord": {"center": [17.3, 11.2, 12.6]}}]
    lbm = LBMD3(config=lbm_config(q, size, 0.06, codes, body_force=[0.0, 2e-6, 0.0],
                                  particles=parts, gl=1e-4, storage=storage))
    f0 = smooth_f0(q, tuple(s + 1 for s in size), 0.02, 900 + q)
    init_with(lbm, f0)
    run(lbm, steps)
    assert lbm.check_status() == 0
    p = lbm.particle_swarm.particles[0]
    return (to64(lbm.flow.rou), to64(lbm.flow.u), to64(p.cx), to64(p.cu))


@pytest.mark.parametrize("q", [19, 27])
def test_storages_vs_fp64_walled_forced_particles(q):
    """fp32, fp16s and bf16s against the FP64 storage on walls + periodic
    faces, a body force and a sphere, 300 steps."""
    steps = 300
    ref = _sphere_run(q, "fp64", steps)
    bounds = {"fp32": 1e-5, "fp16s": 1e-3, "bf16s": 2e-2}
    for storage, bound in bounds.items():
        rou, u, cx, cu = _sphere_run(q, storage, steps)
        e_rho = rel(rou, ref[0])
        e_u = np.abs(u - ref[1]).max() / np.abs(ref[1]).max()
        e_cx = np.abs(cx - ref[2]).max()
        e_cu = np.abs(cu - ref[3]).max()
        print("D3Q%d %s vs fp64 after %d steps: rho %.2e, u %.2e, cx %.2e, cu %.2e"
              % (q, storage, steps, e_rho, e_u, e_cx, e_cu))
        assert e_rho <= bound and e_u <= bound, storage
        if storage != "bf16s":
            assert e_cx <= 1e-4 and e_cu <= 1e-4, storage
