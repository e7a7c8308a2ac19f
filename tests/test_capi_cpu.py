"""C-ABI checks that need no GPU: the library loads, exports every function
declared in include/*.h, and validates lattice descriptions the way the
reference's API raises (ValueError / NotImplementedError)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from funlbm_b200 import _lib
from funlbm_b200.config import BoundaryCondition
from funlbm_b200.lbm import Config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(\w+)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "sizeof", "return"):
                names.add(name)
    return names


@pytest.fixture(scope="module")
def lib():
    from funlbm_b200 import build

    build.build()
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    declared = _declared_functions()
    assert len(declared) >= 14
    for name in declared:
        assert hasattr(lib, name), name
    assert set(_lib.SIGNATURES) >= declared - set(), declared - set(_lib.SIGNATURES)


def test_version_and_error_channel(lib):
    assert b"sm_100a" in lib.lbm_version()


def _desc(q=19, shape=(5, 6, 7), faces=(1200,) * 6, tau=0.8):
    d = _lib.LbmLattice()
    d.q = q
    d.nx, d.ny, d.nz = shape
    for i, c in enumerate(faces):
        d.face[i] = c
    d.tau = tau
    d.cs2 = 1.0 / 3
    return d


def test_lattice_check_codes(lib):
    ok = _desc()
    assert lib.lbm_lattice_check(ctypes.byref(ok)) == _lib.LBM_OK
    bad_q = _desc(q=17)
    assert lib.lbm_lattice_check(ctypes.byref(bad_q)) == _lib.LBM_ERR_INVALID
    assert b"D3Q17" in lib.lbm_last_error()
    bad_tau = _desc(tau=0.5)
    assert lib.lbm_lattice_check(ctypes.byref(bad_tau)) == _lib.LBM_ERR_INVALID
    # y/z faces accept PERIODICAL / WALL / WALL_WITH_SPEED only (flow/d3/base.py:262-263)
    neq_y = _desc(faces=(1200, 1200, 1400, 1200, 1200, 1200))
    assert lib.lbm_lattice_check(ctypes.byref(neq_y)) == _lib.LBM_ERR_UNSUPPORTED
    far = _desc(faces=(1300, 1200, 1200, 1200, 1200, 1200))
    assert lib.lbm_lattice_check(ctypes.byref(far)) == _lib.LBM_ERR_UNSUPPORTED
    with pytest.raises(NotImplementedError):
        _lib.check(lib.lbm_lattice_check(ctypes.byref(far)))
    # NON_EQUILIBRIUM input needs its inlet profile
    neq_x = _desc(faces=(1400, 1200, 1200, 1200, 1200, 1200))
    assert lib.lbm_lattice_check(ctypes.byref(neq_x)) == _lib.LBM_ERR_INVALID
    huge = _desc(shape=(2048, 2048, 1024))
    assert lib.lbm_lattice_check(ctypes.byref(huge)) == _lib.LBM_ERR_INVALID


def test_face_plane_size(lib):
    d = _desc(shape=(5, 6, 7))
    assert lib.lbm_face_plane_floats(ctypes.byref(d)) == 2 * (6 * 7 + 5 * 7 + 5 * 6)


def test_fastdiv_formula():
    """The node-index division used by every kernel: m = ceil(2^(31+l)/d),
    q = (n * m) >> (31 + l) equals n // d for all n < 2^31."""
    rng = np.random.default_rng(0)
    for d in list(range(1, 70)) + [127, 128, 129, 511, 512, 513, 1000, 4097, 65535, 65537,
                                   2 ** 20 + 7, 2 ** 30 + 3]:
        if d == 1:
            continue
        l = (d - 1).bit_length()
        m = -(-(1 << (31 + l)) // d)
        assert m < 2 ** 32
        ns = np.concatenate([rng.integers(0, 2 ** 31, 2000), [0, 1, d - 1, d, d + 1, 2 ** 31 - 1]])
        for n in ns.tolist():
            assert (n * m) >> (31 + l) == n // d, (n, d)


def test_config_parsing_matches_reference_rules():
    cfg = Config().from_json({
        "dt": 0, "flow": {"size": [8, 9, 10], "param_type": "D3Q27",
                          "param": {"mu": 0.1, "Re": 0, "gl": 2e-5},
                          "boundary": {"input": {"code": "PERIODICAL"}, "top": {"code": 11000},
                                       "bottom": {"code": "NOPE"}, "left": {"code": "PERIODICAL"}}},
        "particles": [{"type": "sphere", "r": 8, "coord": {"center": [1, 2, 3], "alpha": 0}}],
    })
    assert cfg.dt == 1.0                                     # 0 -> default (x or default)
    fc = cfg.flow_config
    assert fc.param_type == "D3Q27" and fc.mu == 0.1 and fc.Re == 10 and fc.gl == 2e-5
    b = fc.boundary
    assert b.input.condition == BoundaryCondition.PERIODICAL
    assert b.top.condition == BoundaryCondition.PERIODICAL  # by value
    assert b.bottom.condition == BoundaryCondition.WALL     # unknown -> WALL
    assert b.output.condition == BoundaryCondition.WALL     # unrecognised key 'left' ignored
    pc = cfg.particles[0]
    assert pc.type == "sphere"
    assert abs(pc.coord_config.alpha - np.pi / 2) < 1e-12    # alpha: 0 -> default pi/2


def test_gpu_required_without_cuda():
    import torch

    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    from funlbm_b200.lbm import LBMD3

    with pytest.raises(RuntimeError):
        LBMD3(config=Config().from_json({"flow": {"size": [4, 4, 4]}}))


def test_normal_build_has_no_bounds_counters(lib):
    """Only the bounds-checked build (FUNLBM_B200_CHECKED=1) counts index
    violations; the normal library says so with -1."""
    assert lib.lbm_debug_bounds_faults(0) == -1


def test_claiming_spread_pair_rejects_missing_buffers(lib):
    """ibm_interpolate_wall_claim / ibm_spread_claimed validate their
    arguments before touching the device: without the field, chunk flags or
    claim array they return LBM_ERR_INVALID with a message naming the call."""
    lat = _desc()
    pt = _lib.LbmParticles()
    dummy = ctypes.c_void_p(16)      # never dereferenced: validation fails first
    rc = lib.ibm_interpolate_wall_claim(ctypes.byref(lat), dummy, None, None, ctypes.byref(pt),
                                        1.0, 1.0, 0, None, dummy, None, dummy, None)
    assert rc == _lib.LBM_ERR_INVALID
    assert b"ibm_interpolate_wall_claim" in lib.lbm_last_error()
    rc = lib.ibm_spread_claimed(ctypes.byref(lat), ctypes.byref(pt), dummy, dummy, None, None)
    assert rc == _lib.LBM_ERR_INVALID
    assert b"ibm_spread_claimed" in lib.lbm_last_error()
    rc = lib.ibm_interpolate_wall_claim(ctypes.byref(lat), dummy, None, None, ctypes.byref(pt),
                                        0.0, 1.0, 0, None, dummy, dummy, dummy, None)
    assert rc == _lib.LBM_ERR_INVALID
    assert b"dt must be positive" in lib.lbm_last_error()
