"""GPU checks of the observation side of the driver: the fused step
statistics behind the per-step log (lbm/base.py:105-144,
flow/base.py:183-206), the asynchronous step log and its SQLite records, a
checkpoint saved and loaded mid-run (lbm/base.py:198-227), and the headless
VTK / Tecplot output of save_bak (lbm/lbm3d.py:169-244).
"""
import json
import logging
import os
import sqlite3

import numpy as np
import pytest

from tests.gpu_util import init_with, lbm_config, require_cuda, run, smooth_f0

pytestmark = pytest.mark.gpu
FACES = ("input", "output", "back", "forward", "bottom", "top")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    require_cuda()


def _torch_stats(lbm):
    vals = []
    for t in (lbm.flow.f, lbm.flow.u, lbm.flow.rou):
        t = t.double()
        vals += [float(t.min()), float(t.mean()), float(t.max())]
    return np.array(vals)


@pytest.mark.parametrize("storage", ["fp32", "fp16s", "fp64"])
def test_step_stats_match_materialised_fields(storage):
    """lbm_flow_stats (one read of the populations, 9 numbers out) gives the
    min / max of the materialised end-of-step f, u, rho exactly and their
    means to 1e-9 relative, with walls, a moving wall, a body force and a
    particle."""
    from funlbm_b200.lbm import LBMD3

    size = (21, 14, 17)
    parts = [{"type": "sphere", "r": 3, "rou": 1.4, "coord": {"center": [10.2, 7.1, 8.3]}}]
    codes = [1200, 1200, 11000, 11000, 1201, 1200]
    uw = np.zeros((6, 3), np.float32)
    uw[4] = (0.01, 0.0, -0.005)
    lbm = LBMD3(config=lbm_config(19, size, 0.08, codes, uw, body_force=[1e-5, 0, 0],
                                  particles=parts, gl=1e-3, storage=storage))
    init_with(lbm, smooth_f0(19, tuple(s + 1 for s in size), 0.03, 5))
    run(lbm, 7)
    fast = lbm.flow.step_stats().cpu().numpy()
    assert lbm.flow._obs_valid is False          # nothing was materialised
    slow = _torch_stats(lbm)
    for k in (0, 2, 3, 5, 6, 8):
        assert fast[k] == slow[k], (k, fast[k], slow[k])
    for k in (1, 4, 7):
        assert abs(fast[k] - slow[k]) <= 1e-9 * max(abs(slow[k]), 1e-12), (k, fast[k], slow[k])
    j = lbm.flow.to_json()
    assert set(j) == {"f", "u", "rho"} and len(j["u"]) == 3


def test_async_step_log_lines_and_store(tmp_path):
    """run() with a logging cadence: every logged step produces the
    reference's line (step, f / u / rho min,mean,max, the particle's state)
    from the device reductions, and a SQLite record with the reference's
    table layout."""
    from funlbm_b200.lbm import LBMD3, Config

    db = str(tmp_path / "steps.db")
    cfg = Config().from_json({
        "device": "cuda", "max_step": 30, "log_per_steps": 10, "graph_steps": 4,
        "file": {"per_steps": 10 ** 9}, "log": {"db": db},
        "flow": {"size": [16, 12, 14], "param_type": "D3Q19", "param": {"mu": 0.1, "gl": 1e-3},
                 "boundary": {k: {"code": "WALL"} for k in FACES}},
        "particles": [{"type": "sphere", "r": 2.5, "rou": 1.3,
                       "coord": {"center": [8.0, 6.0, 7.0]}}]})
    lines = []

    class Grab(logging.Handler):
        def emit(self, record):
            lines.append(record.getMessage())

    log = logging.getLogger("funlbm_b200")
    h = Grab()
    old = log.level
    log.addHandler(h)
    log.setLevel(logging.INFO)
    try:
        lbm = LBMD3(config=cfg)
        lbm.run()
    finally:
        log.removeHandler(h)
        log.setLevel(old)
    steps = [ln for ln in lines if ln.startswith("step=")]
    assert len(steps) == 3
    last = steps[-1].split("\t")
    assert last[0] == "step=%6d" % 30
    rho = [float(v) for v in last[3][len("rho="):].split(",")]
    ref = _torch_stats(lbm)
    assert np.allclose(rho, ref[6:9], atol=2e-6)
    assert last[4].startswith("m=")
    con = sqlite3.connect(db)
    rows = dict(con.execute("SELECT key, value FROM flow").fetchall())
    assert sorted(int(k) for k in rows) == [10, 20, 30]
    assert np.allclose(json.loads(rows["30"])["rho"], ref[6:9], atol=2e-6)
    prow = con.execute("SELECT value FROM particle WHERE key1 = '30' AND key2 = '1'").fetchone()
    p = lbm.particle_swarm.particles[0]
    assert np.allclose(json.loads(prow[0])["cx"], p.cx.double().cpu().numpy(), atol=1e-6)
    con.close()


def test_checkpoint_round_trip_continues_identically(tmp_path):
    """Save at step 20 (run_step's cadence), load into a fresh LBMD3 and run
    20 more steps: the state equals 40 uninterrupted steps bit for bit,
    particle rotation vector included (the reference saves no angle and its
    load raises TypeError: lbm/base.py:198-227, base/work.py:60-63).  Like
    the reference, a loaded run resumes with the saved step's number, so the
    test advances the counter by one before continuing."""
    from funlbm_b200.lbm import LBMD3, Config

    def cfg(**extra):
        d = {"device": "cuda", "log_per_steps": 10 ** 9, "graph_steps": 8,
             "file": {"per_steps": 20, "cache_dir": str(tmp_path)},
             "flow": {"size": [20, 14, 16], "param_type": "D3Q19",
                      "param": {"mu": 0.08, "gl": 2e-3}, "body_force": [0.0, 3e-6, 0.0],
                      "boundary": {k: {"code": "WALL"} for k in FACES}},
             "particles": [{"type": "ellipsoid", "a": 3, "b": 2.5, "c": 2, "rou": 1.3,
                            "coord": {"center": [10.2, 7.1, 8.4], "alpha": 0.4,
                                      "beta": 0.2, "gamma": 0.1}}]}
        d.update(extra)
        return Config().from_json(d)

    def state(lbm):
        p = lbm.particle_swarm.particles[0]
        return [t.detach().cpu().numpy().copy() for t in
                (lbm.flow.rou, lbm.flow.u, p.cx, p.cu, p.cw, p.coord.angle, p.lx)]

    a = LBMD3(config=cfg(file={"per_steps": 10 ** 9, "cache_dir": str(tmp_path / "a")}))
    a.init()
    a.run_steps(40)
    ref = state(a)
    b = LBMD3(config=cfg())
    b.init()
    b.run_steps(20)
    ckpt = [f for f in os.listdir(os.path.join(tmp_path, "checkpoint")) if "0000000020" in f]
    assert len(ckpt) == 1
    c = LBMD3(config=cfg(checkpoint=os.path.join(tmp_path, "checkpoint", ckpt[0]),
                         file={"per_steps": 10 ** 9, "cache_dir": str(tmp_path / "c")}))
    c.init()
    assert c.step == 20
    c.step += 1
    c.run_steps(20)
    got = state(c)
    for k, (x, y) in enumerate(zip(got, ref)):
        assert np.array_equal(x, y), k


def test_save_bak_writes_vtk_and_tecplot(tmp_path):
    from funlbm_b200.lbm import LBMD3, Config

    cfg = Config().from_json({
        "device": "cuda", "log_per_steps": 10 ** 9,
        "file": {"per_steps": 5, "cache_dir": str(tmp_path)},
        "flow": {"size": [9, 7, 8], "param_type": "D3Q19", "param": {"mu": 0.1},
                 "body_force": [1e-5, 0, 0],
                 "boundary": {k: {"code": "PERIODICAL"} for k in FACES}},
        "particles": [{"type": "sphere", "r": 2, "coord": {"center": [5.0, 4.0, 4.0]}}]})
    lbm = LBMD3(config=cfg)
    lbm.init()
    lbm.run_steps(5)
    lbm.save_bak(5)
    lbm.flush_output()
    s = "0000000005"
    vtk = tmp_path / "vtk" / ("flow_%s.vtk" % s)
    tec = tmp_path / "tecplot" / ("tecplot_flow_u_%s.dat" % s)
    part = tmp_path / "vtk" / ("particle_000_%s.vtk" % s)
    assert vtk.exists() and tec.exists() and part.exists()
    u = lbm.flow.u.cpu().numpy()
    raw = vtk.read_bytes()
    head = raw.index(b"VECTORS u float\n") + len(b"VECTORS u float\n")
    X, Y, Z = u.shape[:3]
    got = np.frombuffer(raw[head:head + X * Y * Z * 12], ">f4").reshape(Z, Y, X, 3)
    assert np.array_equal(got.transpose(2, 1, 0, 3), u)
    lines = tec.read_text().splitlines()
    assert lines[2] == "ZONE I=%d, J=%d, K=%d, F=POINT" % (X, Y, Z)
    row = lines[3 + 1].split()                 # node x=1, y=0, z=0
    assert [int(v) for v in row[:3]] == [1, 0, 0]
    assert np.allclose([float(v) for v in row[3:]], u[1, 0, 0], rtol=1e-6, atol=1e-12)
