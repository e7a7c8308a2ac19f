"""GPU parity of the immersed-boundary + rigid-particle path against the
reference's recorded particle runs and the oracle.

Tolerance: particle position / velocity / angular velocity / rotation vector
within 1e-4 (lattice units, or relative to the magnitude when it exceeds 1);
marker force lF within 1e-4 relative to its maximum; force / torque sums
within 1e-3 relative (the kernel sums in float64, the reference in float32
over hundreds of markers); flow fields within 2e-5 relative.
"""
import os
import sys

import numpy as np
import pytest
import torch

from oracle import lbm_oracle as O
from tests.gpu_util import init_with, lbm_config, rel_err, require_cuda, run, to_np

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
sys.path.insert(0, GOLD)
from make_golden import PARTICLE_CASES  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    require_cuda()


def _codes(face):
    return [{"WALL": 1200, "PERIODICAL": 11000}[face]] * 6


def _make(case, fused=True, ibm_mode="reference"):
    from funlbm_b200.lbm import LBMD3

    name, q, size, mu, gl, face, parts, nsteps, amp = case
    lbm = LBMD3(config=lbm_config(q, size, mu, _codes(face), particles=parts, gl=gl, fused=fused,
                                  ibm_mode=ibm_mode))
    return lbm


def _stack(lbm, key):
    ps = lbm.particle_swarm.particles
    if key == "angle":
        return np.stack([to_np(p.coord.angle) for p in ps])
    if key in ("lx", "lF", "lu"):
        return np.concatenate([to_np(getattr(p, key)) for p in ps])
    return np.stack([to_np(getattr(p, key)) for p in ps])


@pytest.mark.parametrize("fused", [True, False], ids=["fused", "reference_sequence"])
@pytest.mark.parametrize("case", PARTICLE_CASES, ids=[c[0] for c in PARTICLE_CASES])
def test_particles_vs_reference(case, fused):
    g = np.load(os.path.join(GOLD, "particles.npz"))
    pre = case[0] + "_"
    lbm = _make(case, fused=fused)
    init_with(lbm, g[pre + "f0"])
    for i, p in enumerate(lbm.particle_swarm.particles):
        # coordinates that are exactly 0 on the surface come out as +-1e-17
        # residues of the crossing solve (closed form here, fsolve there)
        assert np.abs(to_np(p._lagrange) - g[pre + "p%d_lagrange" % i]).max() <= 1e-6
        assert abs(float(p.mass) - g[pre + "masses"][i]) <= 1e-6 * g[pre + "masses"][i]
        assert np.allclose(to_np(p.I), g[pre + "inertia"][i], rtol=1e-6)
    for s in range(case[7]):
        run(lbm, 1)
        for k in ("cx", "cu", "cw", "angle"):
            ref = g[pre + k][s]
            assert np.abs(_stack(lbm, k) - ref).max() <= 1e-4 * max(1.0, np.abs(ref).max()), (s, k)
        for k in ("cF", "cT"):
            ref = g[pre + k][s]
            assert np.abs(_stack(lbm, k) - ref).max() <= 1e-3 * max(1.0, np.abs(ref).max()), (s, k)
        for k in ("lx", "lu"):
            ref = g[pre + k][s]
            assert np.abs(_stack(lbm, k) - ref).max() <= 1e-4 * max(1.0, np.abs(ref).max()), (s, k)
        ref = g[pre + "lF"][s]
        assert np.abs(_stack(lbm, "lF") - ref).max() <= 1e-4 * np.abs(ref).max(), s
        if s == 0:
            ref = g[pre + "FOL_first"]
            assert np.abs(to_np(lbm.flow.FOL) - ref).max() <= 1e-4 * np.abs(ref).max()
    for k, attr in (("FOL", "FOL"), ("u", "u"), ("rou", "rou")):
        ref = g[pre + k + "_last"]
        got = to_np(getattr(lbm.flow, attr))
        assert np.abs(got - ref).max() <= 2e-5 * max(np.abs(ref).max(), 1e-3), k


def _oracle_case(case, g, ibm_mode="reference", nsteps=None):
    name, q, size, mu, gl, face, parts, steps, amp = case
    pre = name + "_"
    fl = O.OracleFlow(q, size, mu, dict(zip(O.FACES, _codes(face))))
    ps = []
    for i, pc in enumerate(parts):
        c = pc["coord"]
        ang = [c.get("alpha") or np.pi / 2, c.get("beta") or 0, c.get("gamma") or 0]
        ps.append(O.OracleParticle(g[pre + "p%d_lagrange" % i], g[pre + "masses"][i],
                                   g[pre + "areas"][i], g[pre + "inertia"][i], pc.get("rou", 1.0),
                                   c["center"], ang))
    lbm = O.OracleLBM(fl, ps, gl=gl, ibm_mode=ibm_mode)
    lbm.init(g[pre + "f0"])
    lbm.run(steps if nsteps is None else nsteps)
    return lbm


def test_accumulate_mode_vs_oracle():
    """ibm.mode = accumulate: spread contributions are summed (atomics) instead
    of assigned.  With the reference's direct-forcing law (lF = 2 rho (U - u) /
    dt on overlapping 4^3 stencils) summed spreading over-corrects and the run
    diverges within about three steps -- in the oracle as on the GPU -- so the
    kernel is checked over the first two steps, markers placed on the body
    before step 1."""
    g = np.load(os.path.join(GOLD, "particles.npz"))
    case = PARTICLE_CASES[2]
    lbm = _make(case, ibm_mode="accumulate")
    init_with(lbm, g[case[0] + "_f0"])
    lbm.particle_swarm.update()
    ref = _oracle_case(case, g, ibm_mode="accumulate", nsteps=0)
    for p in ref.particles:
        p.update()
    assert np.abs(_stack(lbm, "lx") - np.concatenate([p.lx for p in ref.particles])).max() < 1e-5
    for s in range(2):
        run(lbm, 1)
        ref.run_step()
        ref.step += 1
        for k in ("cx", "cu", "cw"):
            got = _stack(lbm, k)
            want = np.stack([getattr(p, k) for p in ref.particles])
            assert np.abs(got - want).max() <= 1e-4 * max(1.0, np.abs(want).max()), (s, k)
        lf = np.concatenate([p.lF for p in ref.particles])
        assert np.abs(_stack(lbm, "lF") - lf).max() <= 1e-4 * np.abs(lf).max(), s
        fol = ref.flow.FOL
        assert np.abs(to_np(lbm.flow.FOL) - fol).max() <= 1e-4 * np.abs(fol).max(), s
        assert rel_err(to_np(lbm.flow.rou), ref.flow.rou) < 2e-5


def test_reference_mode_is_deterministic():
    """Last-writer-wins spreading resolves by marker order, not by timing: two
    runs agree bit for bit."""
    g = np.load(os.path.join(GOLD, "particles.npz"))
    case = PARTICLE_CASES[2]
    outs = []
    for _ in range(2):
        lbm = _make(case)
        init_with(lbm, g[case[0] + "_f0"])
        run(lbm, 6)
        outs.append((to_np(lbm.flow.f), _stack(lbm, "cx"), to_np(lbm.flow.FOL)))
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_sphere_freefall_longer_vs_oracle():
    """A sphere sedimenting under gravity in a closed box, 60 steps, against the
    oracle: trajectory within 1e-4 lattice units."""
    from funlbm_b200.lbm import LBMD3

    size = (40, 24, 24)
    parts = [{"type": "sphere", "r": 4, "rou": 1.5, "coord": {"center": [28, 12, 12]}}]
    lbm = LBMD3(config=lbm_config(19, size, 1.0 / 15, [1200] * 6, particles=parts, gl=2e-4))
    init_with(lbm, None)
    run(lbm, 60)
    p = lbm.particle_swarm.particles[0]
    fl = O.OracleFlow(19, size, 1.0 / 15, dict(zip(O.FACES, [1200] * 6)))
    lag = to_np(p._lagrange)
    op = O.OracleParticle(lag, float(p.mass), float(p.area), to_np(p.I), 1.5, [28, 12, 12],
                          [np.pi / 2, 0, 0])
    ref = O.OracleLBM(fl, [op], gl=2e-4)
    ref.init(None)
    ref.run(60)
    assert np.abs(to_np(p.cx) - op.cx).max() <= 1e-4
    assert np.abs(to_np(p.cu) - op.cu).max() <= 1e-4
    assert np.abs(to_np(p.cw) - op.cw).max() <= 1e-4
    assert rel_err(to_np(lbm.flow.rou), fl.rou) < 2e-5


def test_run_with_graphs_matches_eager():
    """LBMD3.run replays the plain fused steps between logging steps from
    captured CUDA graphs (graph_steps); across the step-100 switch of the
    interpolation check and a logging cadence of 9 the state is bit for bit
    the one of the eager loop (graph_steps = 0)."""
    from funlbm_b200.lbm import LBMD3, Config

    faces = ("input", "output", "back", "forward", "bottom", "top")

    def cfg(graph_steps):
        return {"device": "cuda", "max_step": 117, "log_per_steps": 9, "graph_steps": graph_steps,
                "file": {"per_steps": 10 ** 9},
                "flow": {"size": [30, 20, 22], "param_type": "D3Q19",
                         "param": {"mu": 0.08, "gl": 1e-3},
                         "boundary": {k: {"code": "WALL"} for k in faces}},
                "particles": [{"type": "sphere", "r": 3, "rou": 1.3,
                               "coord": {"center": [14.0, 10.0, 11.0]}}]}

    out = []
    for gs in (0, 8):
        lbm = LBMD3(config=Config().from_json(cfg(gs)))
        lbm.run()
        assert lbm.step == 117 and lbm.status_word == 0
        p = lbm.particle_swarm.particles[0]
        out.append((to_np(lbm.flow.rou), to_np(lbm.flow.u), to_np(p.cx), to_np(p.cw)))
        if gs:
            assert len(lbm._graphs) >= 2          # before and after step 100
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("storage", ["fp32", "fp64"])
def test_fused_particle_calls_match_separate_calls(storage):
    """ibm_interpolate_wall + rigid_step (the driver's calls) against
    ibm_interpolate + rigid_wall_and_update(RIGID_WALL | RIGID_UPDATE) +
    rigid_update_markers (one reference function each) on the same state:
    forces, particle state, rotation vectors and new marker positions agree
    bit for bit, and the extremes rigid_step leaves are those of the new
    positions.  Particles touch the walls (the spring acts) and one has
    duplicate extreme markers (a tiny sphere)."""
    import ctypes

    from funlbm_b200 import _lib
    from funlbm_b200._lib import call, ptr
    from funlbm_b200.lattice import ctypes_ref, make_force

    dt = torch.float64 if storage == "fp64" else torch.float32
    parts = [{"type": "sphere", "r": 3, "rou": 1.4, "coord": {"center": [2.2, 8.0, 9.1]}},
             {"type": "ellipsoid", "a": 3, "b": 2, "c": 2.5, "rou": 0.7,
              "coord": {"center": [14.5, 13.3, 1.6], "alpha": 0.3, "beta": -0.5, "gamma": 0.2}},
             {"type": "sphere", "r": 1, "rou": 1.1, "coord": {"center": [9.0, 6.0, 9.0]}}]
    states = []
    for variant in ("separate", "fused"):
        lbm = LBMD3_with(parts, storage)
        lat = lbm.flow.lattice
        sw = lbm.particle_swarm
        sw.update()                               # markers on the bodies
        g = torch.Generator(device="cpu").manual_seed(3)
        sw.cu.copy_((0.01 * torch.randn(sw.cu.shape, generator=g)).to(dt))
        sw.cw.copy_((0.01 * torch.randn(sw.cw.shape, generator=g)).to(dt))
        st = ctypes.byref(sw.struct())
        s = lat.stream()
        force = make_force()
        status = torch.zeros(1, dtype=torch.int32, device="cuda")
        if variant == "separate":
            call("ibm_interpolate", ctypes_ref(lat.desc), ptr(lat.buf[lat.cur]), ctypes_ref(force),
                 ptr(lat.face_rho[lat.cur]), None, None, st, 1.0, 5, ptr(status), s)
            call("rigid_wall_and_update", ctypes_ref(lat.desc), st,
                 _lib.RIGID_WALL | _lib.RIGID_UPDATE, 1.0, 1.0, 1e-3, 1.0, s)
            call("rigid_update_markers", st, s)
            ext = None
        else:
            call("rigid_extremes", st, s)
            call("ibm_interpolate_wall", ctypes_ref(lat.desc), ptr(lat.buf[lat.cur]),
                 ctypes_ref(force), ptr(lat.face_rho[lat.cur]), st, 1.0, 1.0, 5, ptr(status), s)
            call("rigid_step", st, 1.0, 1e-3, 1.0, s)
            ext = sw.extreme.cpu().numpy()[:len(parts)]
        torch.cuda.synchronize()
        states.append([t.cpu().numpy().copy() for t in
                       (sw.lF, sw.lu, sw.cF, sw.cT, sw.cx, sw.cu, sw.cw, sw.angle, sw.lx)])
        if ext is not None:
            lx = sw.lx.cpu().numpy()
            offs = sw._offsets_host
            for i in range(len(parts)):
                seg = lx[offs[i]:offs[i + 1]]
                want = np.concatenate([np.argmin(seg, 0), np.argmax(seg, 0)]) + offs[i]
                assert np.array_equal(ext[i], want), i
    spring = np.abs(states[1][0] - states[0][0]).max()
    for k, (a, b) in enumerate(zip(*states)):
        assert np.array_equal(a, b), (k, np.abs(a - b).max(), spring)


@pytest.mark.parametrize("storage", ["fp32", "fp64"])
def test_claiming_interpolation_matches_interpolation_and_spread(storage):
    """ibm_interpolate_wall_claim + ibm_spread_claimed (the driver's calls in
    reference mode) against ibm_interpolate_wall + ibm_spread(mode 0): the
    same marker forces and velocities, field and chunk flags bit for bit, and
    the claim array back at -1, on two calls in a row (the second clears what
    the first wrote, after the particles have moved).  Particles touch the
    walls, so the spring and stencils cut by the lattice's faces take part."""
    import ctypes

    from funlbm_b200._lib import call, ptr
    from funlbm_b200.lattice import ctypes_ref, make_force

    dt = torch.float64 if storage == "fp64" else torch.float32
    parts = [{"type": "sphere", "r": 3, "rou": 1.4, "coord": {"center": [2.2, 8.0, 9.1]}},
             {"type": "ellipsoid", "a": 3, "b": 2, "c": 2.5, "rou": 0.7,
              "coord": {"center": [14.5, 13.3, 1.6], "alpha": 0.3, "beta": -0.5, "gamma": 0.2}},
             {"type": "sphere", "r": 2, "rou": 1.1, "coord": {"center": [9.0, 6.0, 9.0]}}]
    lbm = LBMD3_with(parts, storage)
    lat = lbm.flow.lattice
    sw = lbm.particle_swarm
    sw.update()
    n = lat.n
    nch = (n + 31) // 32
    bufs = {v: (torch.zeros(3 * n, device="cuda", dtype=dt),
                torch.zeros(nch, dtype=torch.uint8, device="cuda"),
                torch.full((n,), -1, dtype=torch.int32, device="cuda"))
            for v in ("plain", "claimed")}
    force = make_force()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = lat.stream()
    for rep in range(2):
        if rep:
            sw.cx.add_(torch.tensor([0.37, -0.21, 0.44], device="cuda", dtype=dt))
            sw.update()
        out = {}
        for v in ("plain", "claimed"):
            field, chunks, owner = bufs[v]
            st = ctypes.byref(sw.struct())
            call("rigid_extremes", st, s)
            args = (ctypes_ref(lat.desc), ptr(lat.buf[lat.cur]), ctypes_ref(force),
                    ptr(lat.face_rho[lat.cur]), st, 1.0, 1.0, 5, ptr(status))
            if v == "plain":
                call("ibm_interpolate_wall", *args, s)
                call("ibm_spread", ctypes_ref(lat.desc), st, 0, ptr(field), ptr(chunks),
                     ptr(owner), s)
            else:
                call("ibm_interpolate_wall_claim", *args, ptr(field), ptr(chunks), ptr(owner), s)
                call("ibm_spread_claimed", ctypes_ref(lat.desc), st, ptr(field), ptr(chunks),
                     ptr(owner), s)
            torch.cuda.synchronize()
            out[v] = [t.cpu().numpy().copy() for t in (sw.lF, sw.lu, field, chunks, owner)]
        assert np.abs(out["plain"][2]).max() > 0
        for k, (a, b) in enumerate(zip(out["plain"], out["claimed"])):
            assert np.array_equal(a, b), (rep, k)
        assert (out["claimed"][4] == -1).all()


def LBMD3_with(parts, storage):
    from funlbm_b200.lbm import LBMD3

    lbm = LBMD3(config=lbm_config(19, (16, 16, 18), 0.1, [1200] * 6, particles=parts, gl=1e-3,
                                  storage=storage))
    init_with(lbm, None)
    run(lbm, 3)
    return lbm


@pytest.mark.parametrize("storage", ["fp32", "fp64"])
def test_tiled_spreading_matches_ibm_spread(storage):
    """ibm_spread_tiled (shared-memory tiles) against ibm_spread (global
    claims): the same field bit for bit in reference mode (last writer wins)
    and within 1e-5 of its maximum in accumulate mode (summation order), the
    same chunk flags, on two calls in a row; including a tile whose marker
    list overflows (a dozen coincident spheres: the tile scans every marker)
    and a body against the lattice's last nodes."""
    import ctypes

    from funlbm_b200 import _lib
    from funlbm_b200._lib import ptr
    from funlbm_b200.lattice import Lattice, tau_float32
    from funlbm_b200.particle import ParticleConfig, ParticleSwarm

    dt = torch.float64 if storage == "fp64" else torch.float32
    shape = (30, 26, 28)
    lat = Lattice(19, shape, [1200] * 6, tau_float32(0.1), storage=storage, device="cuda",
                  allocate=False)
    bodies = [(3, [8.0, 9.5, 10.2]), (2.5, [11.3, 12.0, 12.7]), (4, [24.6, 20.4, 22.1])]
    bodies += [(3, [17.2, 6.3, 8.8])] * 12             # one tile sees > 512 markers
    cfgs = [ParticleConfig().from_json({"type": "sphere", "r": r, "coord": {"center": c}})
            for r, c in bodies]
    sw = ParticleSwarm(cfgs, device="cuda", dtype=dt)
    sw.init()
    sw.update()
    n = lat.n
    nch = (n + 31) // 32
    lib = _lib.load()
    nbytes = lib.ibm_spread_tiled_scratch_bytes(ctypes.byref(lat.desc), sw.struct().n_markers)
    scratch = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    for mode in (0, 1):
        fa = torch.zeros(3 * n, device="cuda", dtype=dt)
        fb = torch.zeros(3 * n, device="cuda", dtype=dt)
        ca = torch.zeros(nch, dtype=torch.uint8, device="cuda")
        cb = torch.zeros(nch, dtype=torch.uint8, device="cuda")
        owner = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        for call in range(2):
            if call:
                sw.cx.add_(torch.tensor([0.37, -0.21, 0.44], device="cuda", dtype=dt))
                sw.update()
            g = torch.Generator(device="cpu").manual_seed(10 + call)
            sw.lF.copy_((0.01 * torch.randn(sw.lF.shape, generator=g)).to(dt))
            st = ctypes.byref(sw.struct())
            _lib.call("ibm_spread", ctypes.byref(lat.desc), st, mode, ptr(fa), ptr(ca), ptr(owner),
                      lat.stream())
            _lib.call("ibm_spread_tiled", ctypes.byref(lat.desc), st, mode, ptr(fb), ptr(cb),
                      ptr(scratch), nbytes, lat.stream())
            torch.cuda.synchronize()
            a, b = fa.cpu().numpy(), fb.cpu().numpy()
            assert np.abs(a).max() > 0
            if mode == 0:
                assert np.array_equal(a, b), (call, np.abs(a - b).max())
            else:
                assert np.abs(a - b).max() <= 1e-5 * np.abs(a).max(), call
            assert np.array_equal(ca.cpu().numpy(), cb.cpu().numpy()), (mode, call)
