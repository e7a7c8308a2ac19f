"""GPU parity of the flow path (C ABI through funlbm_b200) against the
reference's golden vectors and the oracle.

Tolerances (float32 throughout, as the reference):
  * single functions vs reference golden: max relative error <= 2e-6;
  * multi-step f, rho: max relative error <= 1e-5; u: max abs error
    <= 1e-5 * max|u| + 2e-7 (u is a small difference of O(1) sums, so its
    float32 noise is absolute, ~3e-8 per step);
  * 1000 steps: max relative error <= 1e-5 in rho and in u (u normalised by
    max|u|), the bound stated for particle-free cases.
"""
import os

import numpy as np
import pytest
import torch

from oracle import lbm_oracle as O
from tests.gpu_util import (init_with, lbm_config, rel_err, require_cuda, run, smooth_f0, to_np)

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    require_cuda()


def _flow(q, size, mu, codes, uw=None, Re=10.0):
    from funlbm_b200.flow import create_flow
    from tests.gpu_util import boundary_json
    from funlbm_b200.flow import FlowConfig

    cfg = FlowConfig().from_json({"size": list(size), "param_type": "D3Q%d" % q,
                                  "param": {"mu": mu, "Re": Re},
                                  "boundary": boundary_json(codes, uw)})
    fl = create_flow(cfg, device="cuda")
    fl.init()
    return fl


def _t(a):
    return torch.tensor(a, device="cuda")


@pytest.mark.parametrize("q", [13, 15, 19, 27])
def test_single_functions_vs_reference(q):
    """cul_equ / f_stream / update_u_rou / cul_equ2, one kernel each, on the
    reference's own random states and face mixes (incl. WALL_WITH_SPEED and
    NON_EQUILIBRIUM)."""
    g = np.load(os.path.join(GOLD, "kat_q%d.npz" % q))
    for c in range(int(g["ncase"])):
        p = "c%d_" % c
        fl = _flow(q, (4, 5, 6), float(g[p + "mu"]), g[p + "faces"], g[p + "uw"], float(g[p + "Re"]))
        fl.f, fl.u, fl.rou, fl.FOL = (_t(g[p + k]) for k in ("f", "u", "rou", "FOL"))
        fl.cul_equ()
        assert rel_err(to_np(fl.f), g[p + "collide_f"]) < 2e-6
        assert rel_err(to_np(fl.feq), g[p + "collide_feq"]) < 2e-6
        fl.f = _t(g[p + "f"])
        fl.f_stream()
        assert rel_err(to_np(fl.f), g[p + "stream_f"]) < 2e-6, (c, g[p + "faces"])
        fl.FOL = _t(g[p + "FOL"])
        fl.update_u_rou()
        assert rel_err(to_np(fl.rou), g[p + "moments_rou"]) < 2e-6
        assert rel_err(to_np(fl.u), g[p + "moments_u"]) < 2e-6
        assert rel_err(to_np(fl.p), g[p + "moments_p"]) < 2e-6
        fl.f, fl.u, fl.FOL = _t(g[p + "f"]), _t(g[p + "u"]), _t(g[p + "FOL"])
        fl.cul_equ2()
        assert rel_err(to_np(fl.f), g[p + "force_f"]) < 2e-6


def _check_state(lbm, ref_f, ref_u, ref_rou):
    f, u, rou = to_np(lbm.flow.f), to_np(lbm.flow.u), to_np(lbm.flow.rou)
    assert rel_err(f, ref_f) < 1e-5
    assert rel_err(rou, ref_rou) < 1e-5
    assert np.abs(u - ref_u).max() <= 1e-5 * np.abs(ref_u).max() + 2e-7


@pytest.mark.parametrize("q", [13, 15, 19, 27])
@pytest.mark.parametrize("fused", [True, False])
def test_run_step_vs_reference(q, fused):
    """LBMD3.run_step sequences recorded from the reference (12 steps,
    PERIODICAL/WALL mixes), fused path and reference call sequence."""
    from funlbm_b200.lbm import LBMD3

    g = np.load(os.path.join(GOLD, "steps_q%d.npz" % q))
    for c in range(int(g["ncase"])):
        p = "c%d_" % c
        lbm = LBMD3(config=lbm_config(q, tuple(g["size"]), float(g[p + "mu"]), g[p + "faces"],
                                      fused=fused))
        init_with(lbm, g[p + "f0"])
        run(lbm, int(g["nsteps"]))
        _check_state(lbm, g[p + "f"], g[p + "u"], g[p + "rou"])


def _oracle_run(q, size, mu, codes, uw, f0, nsteps, body_force=None, dtype=np.float32):
    faces = dict(zip(O.FACES, [int(c) for c in codes]))
    uwd = None if uw is None else {k: uw[i] for i, k in enumerate(O.FACES)}
    fl = O.OracleFlow(q, size, mu, faces, uwd, dtype=dtype)
    lbm = O.OracleLBM(fl, body_force=body_force)
    lbm.init(f0)
    lbm.run(nsteps)
    return fl


@pytest.mark.parametrize("q", [13, 15, 19, 27])
def test_fused_random_faces_vs_oracle(q):
    """Random PERIODICAL / WALL / WALL_WITH_SPEED mixes, with and without a
    body force, ragged shapes, 25 steps."""
    from funlbm_b200.lbm import LBMD3

    rng = np.random.default_rng(q)
    for case in range(3):
        size = tuple(int(v) for v in rng.integers(4, 11, 3))
        shape = tuple(s + 1 for s in size)
        codes = rng.choice([11000, 1200, 1201], 6)
        uw = (0.02 * rng.standard_normal((6, 3))).astype(np.float32)
        bf = None if case == 0 else (1e-5 * rng.standard_normal(3)).tolist()
        mu = float(rng.uniform(0.03, 0.2))
        f0 = smooth_f0(q, shape, 0.04, 10 * q + case)
        lbm = LBMD3(config=lbm_config(q, size, mu, codes, uw, body_force=bf))
        init_with(lbm, f0)
        run(lbm, 25)
        ref = _oracle_run(q, size, mu, codes, uw, f0, 25, body_force=bf)
        _check_state(lbm, ref.f, ref.u, ref.rou)


def test_fused_equals_reference_sequence():
    """The fused kernel and the one-kernel-per-function sequence give the same
    state (only float32 rounding order differs)."""
    from funlbm_b200.lbm import LBMD3

    q, size = 19, (23, 17, 29)
    codes = [1200, 1200, 11000, 11000, 1201, 1200]
    uw = np.zeros((6, 3), np.float32)
    uw[4] = (0.01, -0.02, 0.0)
    f0 = smooth_f0(q, tuple(s + 1 for s in size), 0.05, 3)
    out = []
    for fused in (True, False):
        lbm = LBMD3(config=lbm_config(q, size, 0.07, codes, uw, body_force=[1e-5, 0, -2e-5],
                                      fused=fused))
        init_with(lbm, f0)
        run(lbm, 30)
        out.append((to_np(lbm.flow.f), to_np(lbm.flow.u), to_np(lbm.flow.rou)))
    assert rel_err(out[0][0], out[1][0]) < 2e-6
    assert rel_err(out[0][2], out[1][2]) < 2e-6
    assert np.abs(out[0][1] - out[1][1]).max() < 1e-6 * np.abs(out[1][1]).max() + 1e-7


def test_1000_steps_vs_oracle():
    """The particle-free bound: <= 1e-5 relative in rho and u after 1000
    float32 steps (u normalised by max|u|).  A lid-driven cavity (top face
    WALL_WITH_SPEED, uw = (0.05, 0, 0)) keeps |u| ~ 1.5e-2; undriven cases
    decay to |u| ~ 1e-6 (the reference zeroes u on all six planes), where any
    two float32 implementations differ by more than 1e-5 relative.  For this
    case the float32 oracle itself differs from a float64 run by 6e-6 (u) and
    8e-6 (rho)."""
    from funlbm_b200.lbm import LBMD3

    q, size = 19, (15, 11, 9)
    codes = [1200, 1200, 1200, 1200, 1200, 1201]
    uw = np.zeros((6, 3), np.float32)
    uw[5] = (0.05, 0.0, 0.0)
    f0 = smooth_f0(q, tuple(s + 1 for s in size), 0.01, 1000)
    lbm = LBMD3(config=lbm_config(q, size, 0.1, codes, uw))
    init_with(lbm, f0)
    run(lbm, 1000)
    ref = _oracle_run(q, size, 0.1, codes, uw, f0, 1000)
    u, rou = to_np(lbm.flow.u), to_np(lbm.flow.rou)
    e_rho = rel_err(rou, ref.rou)
    e_u = np.abs(u - ref.u).max() / np.abs(ref.u).max()
    print("1000 steps: rho rel err %.2e, u rel err %.2e, max|u| %.3g" % (e_rho, e_u, np.abs(ref.u).max()))
    assert np.abs(ref.u).max() > 1e-2
    assert e_rho <= 1e-5
    assert e_u <= 1e-5


def test_c_abi_direct_init_and_step():
    """Lattice (raw C ABI): lbm_flow_init with an initial field, fused steps,
    observation -- against the oracle."""
    from funlbm_b200.lattice import Lattice, cs2_float32, make_force, tau_float32

    q, size = 27, (12, 9, 14)
    shape = tuple(s + 1 for s in size)
    codes = [11000, 11000, 1200, 1201, 11000, 11000]
    uw = np.zeros((6, 3), np.float32)
    uw[3] = (0.03, 0.0, -0.01)
    mu = 0.09
    f0 = smooth_f0(q, shape, 0.04, 77)
    lat = Lattice(q, shape, codes, tau_float32(mu), face_uw=uw.tolist(), device="cuda")
    f0_soa = torch.tensor(np.ascontiguousarray(np.moveaxis(f0, -1, 0)), device="cuda")
    lat.init(f0_soa)
    force = make_force((0, 0, 0), (0, 0, 0))
    for _ in range(10):
        lat.step(force)
    f = torch.empty(q * lat.n, device="cuda")
    rho = torch.empty(lat.n, device="cuda")
    u = torch.empty(lat.n * 3, device="cuda")
    lat.observe(force, f=f, rho=rho, u=u)
    torch.cuda.synchronize()
    ref = _oracle_run(q, size, mu, codes, uw, f0, 10)
    f_ref = np.moveaxis(ref.f, -1, 0).reshape(q, -1)
    assert rel_err(to_np(f).reshape(q, -1), f_ref) < 1e-5
    assert rel_err(to_np(rho), ref.rou.reshape(-1)) < 1e-5
    assert np.abs(to_np(u) - ref.u.reshape(-1)).max() <= 1e-5 * np.abs(ref.u).max() + 2e-7
    assert lat.read_status() == 0
    assert abs(cs2_float32() - float(ref.cs2)) == 0.0


def test_periodic_mass_conservation_large():
    """128^3 periodic cube: total mass is conserved to float32 rounding, and the
    velocity field of a Taylor-Green vortex stays finite and decays."""
    from funlbm_b200.lbm import LBMD3

    q, size = 19, (127, 127, 127)
    lbm = LBMD3(config=lbm_config(q, size, 1.0 / 30, [11000] * 6))
    lbm.config.flow_config.init_field = {"type": "taylor_green", "u0": 0.05}
    lbm.init()
    m0 = float(lbm.flow.rou.double().sum())
    ke0 = float((lbm.flow.u.double() ** 2).sum())
    run(lbm, 50)
    m1 = float(lbm.flow.rou.double().sum())
    ke1 = float((lbm.flow.u.double() ** 2).sum())
    assert abs(m1 - m0) / m0 < 1e-5
    assert 0 < ke1 < ke0
    assert lbm.check_status() == 0


def test_status_word_flags_bad_density():
    """A NaN population sets LBM_STATUS_RHO_BAD in the device status word; the
    context stays usable."""
    from funlbm_b200 import _lib
    from funlbm_b200.lbm import LBMD3

    q, size = 19, (7, 7, 7)
    f0 = smooth_f0(q, tuple(s + 1 for s in size), 0.02, 5)
    f0[3, 3, 3, 5] = np.nan
    lbm = LBMD3(config=lbm_config(q, size, 0.1, [11000] * 6))
    init_with(lbm, f0)
    run(lbm, 2)
    word = lbm.check_status()
    assert word & _lib.LBM_STATUS_RHO_BAD
    assert lbm.run_status is False
    lbm2 = LBMD3(config=lbm_config(q, size, 0.1, [11000] * 6))
    init_with(lbm2, smooth_f0(q, tuple(s + 1 for s in size), 0.02, 6))
    run(lbm2, 2)
    assert lbm2.check_status() == 0


def taylor_green_f0(q, shape, u0):
    """f = feq(rho = 1, u_TG) in float32 with the reference's feq formula
    (flow/d3/base.py:152-158); u_TG = u0 (sin kx cos ky cos kz,
    -cos kx sin ky cos kz, 0), k = 2 pi / N per axis."""
    e, w, _ = O.velocity_set(q)
    X, Y, Z = shape
    x = np.arange(X)[:, None, None] * (2 * np.pi / X)
    y = np.arange(Y)[None, :, None] * (2 * np.pi / Y)
    z = np.arange(Z)[None, None, :] * (2 * np.pi / Z)
    ux = u0 * np.sin(x) * np.cos(y) * np.cos(z)
    uy = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
    u = np.stack(np.broadcast_arrays(ux, uy, 0 * ux), -1).astype(np.float32)
    cs2 = O.cs2_of(np.float32)
    tmp = (u @ e.T.astype(np.float32)) / cs2
    u2 = np.sqrt((u * u).sum(-1, keepdims=True)) ** 2 / cs2 / np.float32(2)
    return ((1 + tmp + tmp ** 2 / 2 - u2) * w.astype(np.float32)).astype(np.float32)


def test_init_field_taylor_green():
    """The init_field extension sets f = feq(1, u_TG) after FlowD3.init."""
    from funlbm_b200.flow import FlowConfig, create_flow

    cfg = FlowConfig().from_json({"size": [15, 11, 7], "param_type": "D3Q19",
                                  "init_field": {"type": "taylor_green", "u0": 0.05}})
    fl = create_flow(cfg, device="cuda")
    fl.init()
    ref = taylor_green_f0(19, (16, 12, 8), 0.05)
    assert rel_err(to_np(fl.f), ref) < 1e-6


@pytest.mark.parametrize("storage,bound", [("fp16s", 1e-3), ("bf16s", 2e-2)])
def test_shifted_storage_vs_fp64(storage, bound):
    """FP16 / BF16 deviations from w, collided in float32, against an FP64
    oracle run of the same Taylor-Green case (48^3 periodic, 200 steps).
    Errors: rho relative, u normalised by max|u|."""
    from funlbm_b200.lbm import LBMD3

    q, size = 19, (47, 47, 47)
    shape = tuple(s + 1 for s in size)
    f0 = taylor_green_f0(q, shape, 0.05)
    lbm = LBMD3(config=lbm_config(q, size, 1.0 / 30, [11000] * 6, storage=storage))
    init_with(lbm, f0)
    run(lbm, 200)
    ref = _oracle_run(q, size, 1.0 / 30, [11000] * 6, None, f0.astype(np.float64), 200,
                      dtype=np.float64)
    u, rou = to_np(lbm.flow.u), to_np(lbm.flow.rou)
    e_rho = rel_err(rou, ref.rou)
    e_u = np.abs(u - ref.u).max() / np.abs(ref.u).max()
    print("%s: rho err %.2e, u err %.2e" % (storage, e_rho, e_u))
    assert e_rho <= bound and e_u <= bound


@pytest.mark.parametrize("q", [13, 15, 19, 27])
@pytest.mark.parametrize("storage", ["fp32", "fp16s", "bf16s"])
def test_launch_shapes_agree_bitwise(q, storage):
    """Every launch shape of the fused step (one node per thread; 2 / 4 / 8
    z-nodes per thread moved as vectors with 128 / 256 threads; whole z-rows
    staged in shared memory by TMA bulk copies) gives bit-identical results,
    face rules included."""
    from funlbm_b200.lattice import Lattice, make_force, tau_float32
    from funlbm_b200.tune import CANDIDATES, shape_ok

    rng = np.random.default_rng(100 + q)
    shape = (9, 7, 16)
    codes = [int(c) for c in rng.choice([11000, 1200, 1201], 6)]
    codes[4], codes[5] = 1201, 11000 if q % 2 else 1201
    uw = (0.02 * rng.standard_normal((6, 3))).tolist()
    f0 = smooth_f0(q, shape, 0.04, q)
    f0_soa = torch.tensor(np.ascontiguousarray(np.moveaxis(f0, -1, 0)), device="cuda")
    bits = 32 if storage == "fp32" else 16
    force = make_force((0, 0, 0), (1e-5, -2e-5, 3e-5))
    results = {}
    for nodes, threads in CANDIDATES[bits]:
        if not shape_ok(nodes, shape[2], bits):
            continue
        lat = Lattice(q, shape, codes, tau_float32(0.07), storage=storage, face_uw=uw, device="cuda")
        lat.set_launch_shape(nodes, threads)
        lat.init(f0_soa)
        for _ in range(4):
            lat.step(force)
        f = torch.empty(q * lat.n, device="cuda")
        lat.observe(force, f=f)
        results[(nodes, threads)] = to_np(f)
    assert len(results) >= 4 and (-1, 256) in results
    ref = results[(1, 256)]
    for k, v in results.items():
        assert np.array_equal(v, ref), (k, np.abs(v - ref).max())


@pytest.mark.parametrize("q", [19, 27])
@pytest.mark.parametrize("storage", ["fp32", "fp16s"])
def test_chunked_force_fields_agree_bitwise(q, storage):
    """Force fields present only in some 32-node chunks, as spreading leaves
    them: chunks with a previous and a new field, with only the previous one
    (the second moment pass must drop it from u), with only the new one, and
    none.  Every launch shape -- the forced kernels skip the forcing pass at
    nodes without any force -- gives the same bits."""
    from funlbm_b200.lattice import Lattice, make_force, tau_float32
    from funlbm_b200.tune import CANDIDATES, shape_ok

    shape = (10, 9, 64)
    n = shape[0] * shape[1] * shape[2]
    nch = (n + 31) // 32
    rng = np.random.default_rng(7 + q)
    kind = rng.integers(0, 4, nch)            # 0 none, 1 old only, 2 new only, 3 both
    kind[:4] = [0, 1, 2, 3]
    ch_old = torch.tensor(((kind == 1) | (kind == 3)).astype(np.uint8), device="cuda")
    ch_new = torch.tensor(((kind == 2) | (kind == 3)).astype(np.uint8), device="cuda")
    node_kind = np.repeat(kind, 32)[:n]
    f_old = 1e-4 * rng.standard_normal((n, 3)).astype(np.float32)
    f_new = 1e-4 * rng.standard_normal((n, 3)).astype(np.float32)
    f_old[~np.isin(node_kind, (1, 3))] = 0
    f_new[~np.isin(node_kind, (2, 3))] = 0
    F_old = torch.tensor(f_old.reshape(-1), device="cuda")
    F_new = torch.tensor(f_new.reshape(-1), device="cuda")
    force = make_force((0, 0, 0), (0, 0, 0), F_old, F_new, ch_old, ch_new)
    codes = [1200, 1200, 11000, 11000, 1200, 11000]
    f0 = smooth_f0(q, shape, 0.04, q + 3)
    f0_soa = torch.tensor(np.ascontiguousarray(np.moveaxis(f0, -1, 0)), device="cuda")
    bits = 32 if storage == "fp32" else 16
    results = {}
    for nodes, threads in CANDIDATES[bits]:
        if not shape_ok(nodes, shape[2], bits):
            continue
        lat = Lattice(q, shape, codes, tau_float32(0.07), storage=storage, device="cuda")
        lat.set_launch_shape(nodes, threads)
        lat.init(f0_soa)
        for _ in range(3):
            lat.step(force)
        assert lat.read_status() == 0
        f = torch.empty(q * lat.n, device="cuda")
        lat.observe(force, f=f)
        results[(nodes, threads)] = to_np(f)
    ref = results[(1, 256)]
    assert len(results) >= 4
    for k, v in results.items():
        assert np.array_equal(v, ref), (k, np.abs(v - ref).max())
    # and the fields did act: without them the state differs
    lat = Lattice(q, shape, codes, tau_float32(0.07), storage=storage, device="cuda")
    lat.init(f0_soa)
    for _ in range(3):
        lat.step(None)
    f = torch.empty(q * lat.n, device="cuda")
    lat.observe(None, f=f)
    assert not np.array_equal(to_np(f), ref)


@pytest.mark.parametrize("q", [13, 19, 27])
@pytest.mark.parametrize("storage", ["fp16s", "bf16s"])
def test_odd_rows_agree_bitwise(q, storage):
    """Rows of odd length in 16-bit storage: the pair kernel for odd rows
    (element-wise loads, the last node of a row through the one-node code,
    pairs that straddle a force chunk) gives the same bits as one node per
    thread, with WALL_WITH_SPEED z faces and chunked force fields."""
    from funlbm_b200.lattice import Lattice, make_force, tau_float32

    shape = (10, 9, 15)
    n = shape[0] * shape[1] * shape[2]
    nch = (n + 31) // 32
    rng = np.random.default_rng(11 + q)
    kind = rng.integers(0, 4, nch)
    ch_old = torch.tensor(((kind == 1) | (kind == 3)).astype(np.uint8), device="cuda")
    ch_new = torch.tensor(((kind == 2) | (kind == 3)).astype(np.uint8), device="cuda")
    node_kind = np.repeat(kind, 32)[:n]
    f_old = 1e-4 * rng.standard_normal((n, 3)).astype(np.float32)
    f_new = 1e-4 * rng.standard_normal((n, 3)).astype(np.float32)
    f_old[~np.isin(node_kind, (1, 3))] = 0
    f_new[~np.isin(node_kind, (2, 3))] = 0
    F_old = torch.tensor(f_old.reshape(-1), device="cuda")
    F_new = torch.tensor(f_new.reshape(-1), device="cuda")
    force = make_force((0, 0, 0), (0, 0, 0), F_old, F_new, ch_old, ch_new)
    codes = [1200, 11000, 11000, 1200, 1201, 1201]
    uw = (0.02 * rng.standard_normal((6, 3))).tolist()
    f0 = smooth_f0(q, shape, 0.04, q + 5)
    f0_soa = torch.tensor(np.ascontiguousarray(np.moveaxis(f0, -1, 0)), device="cuda")
    results = {}
    for nodes, threads in [(1, 256), (2, 128), (2, 256)]:
        lat = Lattice(q, shape, codes, tau_float32(0.07), storage=storage, face_uw=uw,
                      device="cuda")
        lat.set_launch_shape(nodes, threads)
        lat.init(f0_soa)
        for _ in range(4):
            lat.step(force)
        assert lat.read_status() == 0
        f = torch.empty(q * lat.n, device="cuda")
        lat.observe(force, f=f)
        results[(nodes, threads)] = to_np(f)
    ref = results[(1, 256)]
    for k, v in results.items():
        assert np.array_equal(v, ref), (k, np.abs(v - ref).max())


def test_row_staged_wait_timeout_sets_status():
    """The row-staged (TMA) step's consumer waits are bounded.  With the test
    hook's limit at zero polls every such wait gives up at once: the kernel
    sets LBM_STATUS_WAIT_TIMEOUT, drains its own bulk copies under the
    default limit (no LBM_STATUS_DRAIN_FAILED) and returns; the context stays
    usable and the default limit steps correctly again."""
    from funlbm_b200 import _lib
    from funlbm_b200.lattice import Lattice, make_force, tau_float32

    q, shape, codes = 19, (9, 7, 16), [11000] * 6
    f0 = smooth_f0(q, shape, 0.04, 21)
    f0_soa = torch.tensor(np.ascontiguousarray(np.moveaxis(f0, -1, 0)), device="cuda")
    force = make_force((0, 0, 0), (0, 0, 0))
    lib = _lib.load()
    lat = Lattice(q, shape, codes, tau_float32(0.07), device="cuda")
    lat.set_launch_shape(-1, 256)
    lat.init(f0_soa)
    lib.lbm_debug_set_wait_limit(0)
    try:
        lat.step(force)
        torch.cuda.synchronize()
    finally:
        lib.lbm_debug_set_wait_limit(-1)
    word = lat.read_status()
    assert word & _lib.LBM_STATUS_WAIT_TIMEOUT
    assert not word & _lib.LBM_STATUS_DRAIN_FAILED
    results = []
    for nodes in (-1, 1):
        lat = Lattice(q, shape, codes, tau_float32(0.07), device="cuda")
        lat.set_launch_shape(nodes, 256)
        lat.init(f0_soa)
        for _ in range(3):
            lat.step(force)
        assert lat.read_status() == 0
        f = torch.empty(q * lat.n, device="cuda")
        lat.observe(force, f=f)
        results.append(to_np(f))
    assert np.array_equal(results[0], results[1])


@pytest.mark.parametrize("storage", ["fp32", "fp16s", "bf16s", "fp64"])
@pytest.mark.parametrize("q", [15, 19, 27])
def test_pitched_rows_agree_bitwise(q, storage):
    """Population rows pitched to the vector width (rows of 13 and 33 nodes
    stored in rows of 16 / 36 / 40 elements): every launch shape on the pitched
    buffers -- vectors over full groups, a partial last vector per row whose
    padding lanes are not finished (or the per-node path under a
    WALL_WITH_SPEED top face) -- gives the bits of one node per thread on
    dense rows, with WALL / PERIODICAL / WALL_WITH_SPEED z faces, walls and
    chunked force fields."""
    from funlbm_b200.lattice import Lattice, make_force, tau_float32
    from funlbm_b200.tune import CANDIDATES, STORAGE_BITS, shape_ok

    rng = np.random.default_rng(50 + q)
    bits = STORAGE_BITS[storage]
    dt = torch.float64 if storage == "fp64" else torch.float32
    for shape, zfaces in (((9, 8, 13), (1201, 1201)), ((7, 6, 33), (1201, 1201)),
                          ((9, 8, 13), (1200, 11000)), ((7, 6, 33), (11000, 1200))):
        n = shape[0] * shape[1] * shape[2]
        nch = (n + 31) // 32
        kind = rng.integers(0, 4, nch)
        ch_old = torch.tensor(((kind == 1) | (kind == 3)).astype(np.uint8), device="cuda")
        ch_new = torch.tensor(((kind == 2) | (kind == 3)).astype(np.uint8), device="cuda")
        node_kind = np.repeat(kind, 32)[:n]
        f_old = 1e-4 * rng.standard_normal((n, 3))
        f_new = 1e-4 * rng.standard_normal((n, 3))
        f_old[~np.isin(node_kind, (1, 3))] = 0
        f_new[~np.isin(node_kind, (2, 3))] = 0
        F_old = torch.tensor(f_old.reshape(-1), device="cuda", dtype=dt)
        F_new = torch.tensor(f_new.reshape(-1), device="cuda", dtype=dt)
        force = make_force((0, 0, 0), (2e-6, 0, 0), F_old, F_new, ch_old, ch_new)
        codes = [1200, 11000, 11000, 1200, *zfaces]
        uw = (0.02 * rng.standard_normal((6, 3))).tolist()
        f0 = smooth_f0(q, shape, 0.04, q + 7)
        f0_soa = torch.tensor(np.ascontiguousarray(np.moveaxis(f0, -1, 0)), device="cuda",
                              dtype=dt)
        results = {}
        for pitch in (False, True):
            for nodes, threads in CANDIDATES[bits]:
                probe = Lattice(q, shape, codes, tau_float32(0.07), storage=storage, face_uw=uw,
                                device="cuda", pitch=pitch, allocate=False)
                if not shape_ok(nodes, probe.pz, bits, shape[2]) or (pitch and nodes == 1):
                    continue
                lat = Lattice(q, shape, codes, tau_float32(0.07), storage=storage, face_uw=uw,
                              device="cuda", pitch=pitch)
                lat.set_launch_shape(nodes, threads)
                lat.init(f0_soa)
                for _ in range(4):
                    lat.step(force)
                assert lat.read_status() == 0
                f = torch.empty(q * lat.n, device="cuda", dtype=dt)
                lat.observe(force, f=f)
                results[(pitch, nodes, threads, lat.pz)] = f.cpu().numpy()
        ref = results[(False, 1, 256, shape[2])]
        assert any(k[0] and k[1] > 1 for k in results)
        for k, v in results.items():
            assert np.array_equal(v, ref), (shape, zfaces, k, np.abs(v - ref).max())
