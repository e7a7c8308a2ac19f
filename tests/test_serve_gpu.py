"""Serving (continuous batching of many lattices) on the GPU: every request's
result is the same alone and in the mix, admission respects the device-memory
budget, and steady phases run from captured CUDA graphs."""
import numpy as np
import pytest
import torch

from tests.gpu_util import require_cuda, to_np

pytestmark = pytest.mark.gpu

FACES = ("input", "output", "back", "forward", "bottom", "top")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    require_cuda()


def _cfg(q, size, faces, storage="fp32", mu=0.08, particles=(), gl=0.0, body=None, tg=None):
    flow = {"size": list(size), "param_type": "D3Q%d" % q, "param": {"mu": mu, "gl": gl},
            "boundary": {k: {"code": c} for k, c in zip(FACES, faces)},
            "precision": {"storage": storage}}
    if body is not None:
        flow["body_force"] = list(body)
    if tg is not None:
        flow["init_field"] = {"type": "taylor_green", "u0": tg}
    return {"device": "cuda", "flow": flow, "particles": list(particles),
            "log_per_steps": 10 ** 9, "file": {"per_steps": 10 ** 9}}


P, W = "PERIODICAL", "WALL"
CASES = [
    (_cfg(19, (23, 19, 27), [P] * 6, tg=0.04), 40),
    (_cfg(27, (17, 15, 21), [W, W, P, P, W, W], body=(0, 0, 2e-5)), 33),
    (_cfg(19, (31, 31, 31), [P] * 6, storage="fp16s", tg=0.05), 26),
    (_cfg(19, (25, 19, 19), [W] * 6, gl=1e-3,
          particles=[{"type": "sphere", "r": 3, "rou": 1.3, "coord": {"center": [12, 9, 9]}},
                     {"type": "sphere", "r": 2.5, "rou": 0.9, "coord": {"center": [18, 10, 10]}}]),
     21),
    (_cfg(15, (16, 14, 18), [P, P, W, W, P, P], tg=0.03), 37),     # nz = 19: one node per thread
    (_cfg(13, (15, 15, 15), [P] * 6, storage="bf16s", tg=0.04), 12),
]


def _alone(cfg, steps):
    from funlbm_b200.lbm import LBMD3, Config

    lbm = LBMD3(config=Config().from_json(dict(cfg)))
    lbm.init()
    for _ in range(steps):
        lbm.run_step(step=lbm.step)
        lbm.step += 1
    out = {"rho": to_np(lbm.flow.rou), "u": to_np(lbm.flow.u)}
    ps = lbm.particle_swarm.particles
    if ps:
        out["cx"] = np.stack([to_np(p.cx) for p in ps])
    return out


@pytest.mark.parametrize("mode", ["streams", "batched"])
def test_results_same_alone_and_in_mix(mode):
    """All requests queued together run on the device at the same time
    (streams: one stream and graph each; batched: one multi-lattice launch per
    class per step); each result equals the request run alone, bit for bit.
    Admission while others run is covered by test_admission_respects_budget."""
    from funlbm_b200.serve import LBMServer, Request

    reqs = [Request(cfg, steps) for cfg, steps in CASES]
    server = LBMServer(budget_bytes=8e9, chunk=8, mode=mode, streams=4)
    if mode == "streams":
        server.prepare(reqs[:2])      # some classes tuned ahead, the rest at admission
    done = server.run(reqs, realtime=False)
    assert len(done) == len(CASES)
    assert server.stats["graph_replays"] > 0 and server.stats["max_active"] == len(CASES)
    for r in reqs:
        ref = _alone(r.config, r.steps)
        got = r.result
        assert got["status"] == 0
        assert got["steps"] == r.steps
        for k in ("rho", "u"):
            # same per-node code in every launch form: identical bits
            assert np.array_equal(to_np(got[k]), ref[k]), (r.rid, k)
        if "cx" in ref:
            assert np.array_equal(to_np(got["cx"]), ref["cx"]), r.rid
        assert r.finished_at is not None and r.finished_at > 0


@pytest.mark.parametrize("mode", ["streams", "batched"])
def test_admission_respects_budget(mode):
    from funlbm_b200.serve import LBMServer, Request, estimate_bytes

    cfgs = [(_cfg(19, (31, 31, 31), [P] * 6, tg=0.03), 10 + 3 * i) for i in range(6)]
    one = estimate_bytes(cfgs[0][0])
    server = LBMServer(budget_bytes=2.5 * one, chunk=4, mode=mode)
    done = server.run([Request(c, s) for c, s in cfgs], realtime=False)
    assert len(done) == 6
    assert server.stats["max_active"] == 2
    assert server.stats["max_used_bytes"] <= 2.5 * one
    with pytest.raises(ValueError):
        server.submit(Request(_cfg(19, (511, 511, 511), [P] * 6), 1))


@pytest.mark.parametrize("mode", ["streams", "batched"])
def test_rejected_request_does_not_stop_the_others(mode):
    """A config the solver refuses (unknown velocity set: ValueError; a
    NON_EQUILIBRIUM z face: NotImplementedError, the reference's error types)
    comes back with the error on its request; the other requests finish with
    the same result as alone."""
    from funlbm_b200.serve import LBMServer, Request

    good_cfg, good_steps = CASES[0]
    bad_q = _cfg(19, (15, 15, 15), [P] * 6)
    bad_q["flow"]["param_type"] = "D3Q17"
    bad_face = _cfg(19, (15, 15, 15), [W, W, W, W, "NON_EQUILIBRIUM", W])
    reqs = [Request(bad_q, 5), Request(good_cfg, good_steps), Request(bad_face, 5)]
    server = LBMServer(budget_bytes=8e9, chunk=8, mode=mode, streams=4)
    done = server.run(reqs, realtime=False)
    assert len(done) == 3 and server.stats["rejected"] == 2
    assert "ValueError" in reqs[0].result["error"]
    assert "NotImplementedError" in reqs[2].result["error"]
    ref = _alone(good_cfg, good_steps)
    assert reqs[1].result["status"] == 0
    for k in ("rho", "u"):
        assert np.array_equal(to_np(reqs[1].result[k]), ref[k]), k
    assert server.used == 0
