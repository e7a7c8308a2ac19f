"""Host-side logic that needs no GPU: launch-shape legality, autotuner class
keys, the server's memory estimate and request bookkeeping, and the config
keys this library adds to the reference's."""
import pytest

from funlbm_b200 import serve, tune
from funlbm_b200.lbm import Config


def test_shape_legality():
    # vectors need rows that are a multiple of their width (and twice as long)
    assert tune.shape_ok(2, 16, 32) and tune.shape_ok(4, 16, 32)
    assert not tune.shape_ok(8, 64, 32)          # 32 bytes per fp32 vector: too wide
    assert tune.shape_ok(8, 64, 16) and not tune.shape_ok(8, 12, 16)
    # rows of odd length: pairs only in 16-bit storage (element-wise pair kernel)
    assert tune.shape_ok(2, 15, 16) and not tune.shape_ok(2, 15, 32)
    assert not tune.shape_ok(4, 15, 16)
    assert tune.shape_ok(1, 15, 32)
    # TMA rows: 16-byte multiples, at least 16 nodes
    assert tune.shape_ok(tune.ROWS, 16, 16) and not tune.shape_ok(tune.ROWS, 12, 32)
    for bits in (16, 32):
        for nodes, _ in tune.CANDIDATES[bits]:
            assert tune.shape_ok(nodes, 512, bits) or nodes == tune.ROWS


def test_class_keys_group_by_row_widths():
    k = tune.class_key_of
    assert k(19, "fp16s", 96, False) == k(19, "fp16s", 160, False)        # both divisible by 8
    assert k(19, "fp16s", 96, False) != k(19, "fp16s", 100, False)        # by 4, not by 8
    assert k(19, "fp16s", 65, False) != k(19, "fp16s", 66, False)         # odd vs even
    assert k(19, "fp16s", 96, False) != k(19, "fp16s", 96, True)          # forced
    assert k(19, "fp16s", 96, False) != k(27, "fp16s", 96, False)
    assert k(19, "fp16s", 96, False) != k(19, "fp32", 96, False)


def _cfg(size, q=19, storage="fp32", particles=()):
    return {"flow": {"size": list(size), "param_type": "D3Q%d" % q,
                     "precision": {"storage": storage}},
            "particles": list(particles)}


def test_memory_estimate():
    e = serve.estimate_bytes
    small, big = e(_cfg((31, 31, 31))), e(_cfg((63, 63, 63)))
    fixed = 8 << 20                                   # per-request allowance
    assert big - fixed > 7 * (small - fixed)          # grows with the node count
    # 16-bit populations take less, more directions take more, particles add IBM buffers
    assert e(_cfg((63, 63, 63), storage="fp16s")) < big
    assert e(_cfg((63, 63, 63), q=27)) > big
    sphere = {"type": "sphere", "r": 4, "coord": {"center": [30, 30, 30]}}
    assert e(_cfg((63, 63, 63), particles=[sphere])) > big
    n = 64 ** 3
    assert big >= 2 * 19 * n * 4                      # at least both population buffers


def test_request_latency_and_refusal_of_oversized():
    r = serve.Request(_cfg((15, 15, 15)), 10, arrival=1.5)
    assert r.latency is None
    r.finished_at = 4.0
    assert r.latency == pytest.approx(2.5)
    assert serve.Request(_cfg((15, 15, 15)), 1).rid != r.rid


def test_added_config_keys():
    c = Config().from_json({})
    assert c.fused is True and c.log_per_steps == 1 and c.graph_steps == 32
    assert c.ibm_mode == "reference"
    c = Config().from_json({"fused": False, "log_per_steps": 50, "graph_steps": 0,
                            "ibm": {"mode": "accumulate"},
                            "flow": {"precision": {"storage": "bf16s"}}})
    assert c.fused is False and c.log_per_steps == 50 and c.graph_steps == 0
    assert c.ibm_mode == "accumulate" and c.flow_config.storage == "bf16s"
    with pytest.raises(ValueError):
        Config().from_json({"ibm": {"mode": "sum"}})


def test_tuner_keeps_the_default_within_its_margin():
    assert tune.default_shape(19, "fp32", 512) == (2, 128)
    assert tune.default_shape(19, "fp16s", 512) == (4, 128)
    assert tune.default_shape(19, "fp16s", 512, forced=True) == (2, 128)
    assert tune.default_shape(27, "bf16s", 514) == (2, 128)
    assert tune.default_shape(19, "fp32", 65) == (1, 256)
    t = {(1, 256): 3.08, (2, 128): 3.10, (4, 128): 3.4}
    assert tune._pick(t, (2, 128)) == (2, 128)          # within 3 %: keep the default
    t[(1, 256)] = 2.9
    assert tune._pick(t, (2, 128)) == (1, 256)          # clearly faster: take it
