"""GPU checks of the FP64 storage (the comparison run of the precision
figures) and of the 16-bit shifted storages against it.

* FP64 storage against the float64 oracle: every velocity set, random
  PERIODICAL / WALL / WALL_WITH_SPEED faces, a body force, ragged shapes, and
  a sedimenting sphere -- the same algorithm, so the two float64 codes agree
  to rounding (max relative error <= 1e-11 in f, rho and u after 25 steps;
  particle position / velocity within 1e-10 lattice units after 60 steps).
* FP32, FP16 and BF16 storage (all three hold f - w_i) against that FP64
  run on walled, forced cases with and without a particle (D3Q19 and
  D3Q27): rho relative and u normalised by max|u| within 1e-4 / 1e-3 / 1e-2
  without the particle, particle position and velocity within 1e-4 lattice
  units for fp32 and fp16s.

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


def _walled_run(q, storage, steps, particle):
    from funlbm_b200.lbm import LBMD3

    size = (30, 22, 25)
    codes = [1200, 1200, 11000, 11000, 1200, 1200]
    parts = ([{"type": "sphere", "r": 4, "rou": 1.3, "coord": {"center": [17.3, 11.2, 12.6]}}]
             if particle else [])
    lbm = LBMD3(config=lbm_config(q, size, 0.06, codes, body_force=[0.0, 2e-6, 0.0],
                                  particles=parts, gl=1e-4, storage=storage))
    f0 = smooth_f0(q, tuple(s + 1 for s in size), 0.02, 900 + q)
    init_with(lbm, f0)
    run(lbm, steps)
    assert lbm.check_status() == 0
    out = [to64(lbm.flow.rou), to64(lbm.flow.u)]
    if particle:
        p = lbm.particle_swarm.particles[0]
        out += [to64(p.cx), to64(p.cu)]
    return out


def _errors_vs_fp64(q, particle, steps=300):
    ref = _walled_run(q, "fp64", steps, particle)
    errs = {}
    for storage in ("fp32", "fp16s", "bf16s"):
        got = _walled_run(q, storage, steps, particle)
        du = np.abs(got[1] - ref[1]).max(axis=3)
        e = {"rho": rel(got[0], ref[0]), "u": float(du.max() / np.abs(ref[1]).max())}
        print("  largest u error at node", np.unravel_index(np.argmax(du), du.shape))
        if particle:
            e["cx"] = float(np.abs(got[2] - ref[2]).max())
            e["cu"] = float(np.abs(got[3] - ref[3]).max())
        print("D3Q%d %s vs fp64, %s, %d steps: %s" % (
            q, storage, "sphere" if particle else "no particle", steps,
            ", ".join("%s %.2e" % kv for kv in e.items())))
        errs[storage] = e
    return errs


@pytest.mark.parametrize("q", [19, 27])
def test_storages_vs_fp64_walled_forced(q):
    """fp32, fp16s and bf16s against the FP64 storage on WALL + PERIODICAL
    faces with a body force, 300 steps: rho relative and u normalised by
    max|u| within 1e-4 (fp32), 1e-3 (fp16s) and 1e-2 (bf16s).  Measured on
    B200 (D3Q19 / D3Q27): rho 6.6e-8 / 6.4e-8, u 4.3e-5 / 4.2e-5 (fp32);
    rho 6.2e-7 / 7.1e-7, u 3.0e-4 / 4.3e-4 (fp16s); rho 4.9e-6 / 3.0e-6,
    u 3.2e-3 / 2.4e-3 (bf16s)."""
    errs = _errors_vs_fp64(q, False)
    for storage, bound in (("fp32", 1e-4), ("fp16s", 1e-3), ("bf16s", 1e-2)):
        assert errs[storage]["rho"] <= bound and errs[storage]["u"] <= bound, storage


@pytest.mark.parametrize("q", [19, 27])
def test_storages_vs_fp64_with_particle(q):
    """The same case with a sphere (IBM forcing, rigid update): particle
    position and velocity within 1e-4 lattice units for fp32 and fp16s.  The
    field bound is wider than without the particle: the reference's
    last-writer-wins spreading gives a node the force of whichever covering
    marker comes last, and a marker whose stencil box moves by one node under
    a rounding difference changes that writer -- a jump of the order of the
    local IBM force, not a rounding-sized difference.  Measured on B200
    (D3Q19 / D3Q27): u 4.5e-5 / 9.8e-5 and cx 2.9e-5 / 1.6e-5 (fp32), u
    3.0e-4 / 3.4e-4 and cx 6.0e-5 / 5.0e-5 (fp16s), u 3.3e-3 / 2.6e-3
    (bf16s)."""
    errs = _errors_vs_fp64(q, True)
    for storage, bound in (("fp32", 3e-4), ("fp16s", 1e-3), ("bf16s", 1e-2)):
        assert errs[storage]["rho"] <= bound and errs[storage]["u"] <= bound, storage
        if storage != "bf16s":
            assert errs[storage]["cx"] <= 1e-4 and errs[storage]["cu"] <= 1e-4, storage
