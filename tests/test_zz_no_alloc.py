"""The allocation-free spreading entry point, ibm_spread_noalloc, against
ibm_spread.

Some callers of this library cannot allocate device memory of their own -- a
solver coupled in through the C ABI that only owns the lattice's buffers, or a
time loop that runs under a fixed device-memory budget.  ibm_spread_noalloc
serves them with a per-node claim array built into the library instead of one
passed in.  These tests call both entry points through the C ABI on the same
markers and forces and require the same spread force field and chunk flags,
on two calls in a row (the built-in array is shared by every call and keeps
what the previous call left), and check that a lattice larger than the
built-in array is refused.

This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from tests.gpu_util import require_cuda, to_np

pytestmark = pytest.mark.gpu

SHAPE = (26, 22, 24)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    require_cuda()


def _lattice(shape=SHAPE):
    from funlbm_b200.lattice import Lattice, tau_float32

    return Lattice(19, shape, [1200] * 6, tau_float32(0.1), device="cuda", allocate=False)


BODIES = ((3, [8.0, 9.5, 10.2]), (2.5, [11.3, 12.0, 12.7]), (4, [17.6, 10.4, 13.1]))


def _swarm(bodies=BODIES):
    from funlbm_b200.particle import ParticleConfig, ParticleSwarm

    cfgs = [ParticleConfig().from_json({"type": "sphere", "r": r, "coord": {"center": c}})
            for r, c in bodies]
    sw = ParticleSwarm(cfgs, device="cuda")
    sw.init()
    sw.update()            # place the markers on the bodies
    return sw


def _forces(sw, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    sw.lF.copy_((0.01 * torch.randn(sw.lF.shape, generator=g)).to(sw.lF.device))


@pytest.mark.parametrize("mode", [0, 1], ids=["reference", "accumulate"])
def test_noalloc_spread_matches_ibm_spread(mode):
    from funlbm_b200 import _lib
    from funlbm_b200._lib import ptr

    lat = _lattice()
    sw = _swarm()
    n = lat.n
    nch = (n + 31) // 32
    field_a = torch.zeros(3 * n, device="cuda")
    chunks_a = torch.zeros(nch, dtype=torch.uint8, device="cuda")
    owner = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    field_b = torch.zeros(3 * n, device="cuda")
    chunks_b = torch.zeros(nch, dtype=torch.uint8, device="cuda")
    stream = lat.stream()
    for call in range(2):
        if call == 1:
            # move the bodies and change the forces before the second call
            sw.cx.add_(torch.tensor([0.61, -0.43, 0.29], device="cuda"))
            sw.update()
        _forces(sw, 100 + call)
        st = ctypes.byref(sw.struct())
        _lib.call("ibm_spread", ctypes.byref(lat.desc), st, mode, ptr(field_a), ptr(chunks_a),
                  ptr(owner), stream)
        _lib.call("ibm_spread_noalloc", ctypes.byref(lat.desc), st, mode, ptr(field_b),
                  ptr(chunks_b), stream)
        torch.cuda.synchronize()
        a, b = to_np(field_a), to_np(field_b)
        assert np.abs(a).max() > 0
        if mode == 0:
            # last-writer-wins: one writer per node, no atomics -- the two
            # entry points run the same deterministic kernels
            assert np.array_equal(a, b), call
        else:
            # accumulation order of the atomics is not deterministic; the
            # tolerance of the spreading comparisons elsewhere in the suite
            assert np.abs(b - a).max() <= 1e-4 * np.abs(a).max(), call
        assert np.array_equal(to_np(chunks_a), to_np(chunks_b)), call
    # the caller-owned claim array is back to its resting value
    assert bool((owner == -1).all())


def test_noalloc_spread_at_the_size_limit():
    """A lattice of exactly LBM_SPREAD_NOALLOC_MAX_NODES nodes is accepted, and
    markers next to its last nodes spread the same field as ibm_spread."""
    from funlbm_b200 import _lib
    from funlbm_b200._lib import ptr

    lat = _lattice((256, 128, 128))
    assert lat.n == _lib.SPREAD_NOALLOC_MAX_NODES
    sw = _swarm(((3, [250.6, 122.3, 123.1]), (2.5, [5.2, 4.4, 3.9])))
    n = lat.n
    nch = (n + 31) // 32
    field_a = torch.zeros(3 * n, device="cuda")
    field_b = torch.zeros(3 * n, device="cuda")
    chunks_a = torch.zeros(nch, dtype=torch.uint8, device="cuda")
    chunks_b = torch.zeros(nch, dtype=torch.uint8, device="cuda")
    owner = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    _forces(sw, 7)
    st = ctypes.byref(sw.struct())
    _lib.call("ibm_spread", ctypes.byref(lat.desc), st, 0, ptr(field_a), ptr(chunks_a), ptr(owner),
              lat.stream())
    _lib.call("ibm_spread_noalloc", ctypes.byref(lat.desc), st, 0, ptr(field_b), ptr(chunks_b),
              lat.stream())
    torch.cuda.synchronize()
    a = to_np(field_a)
    assert np.abs(a[3 * (n // 2):]).max() > 0          # the far body reached the upper half
    assert np.array_equal(a, to_np(field_b))
    assert np.array_equal(to_np(chunks_a), to_np(chunks_b))


def test_noalloc_spread_rejects_large_lattice():
    from funlbm_b200 import _lib
    from funlbm_b200._lib import ptr

    big = _lattice((256, 256, 256))
    assert big.n > _lib.SPREAD_NOALLOC_MAX_NODES
    sw = _swarm()
    field = torch.zeros(3, device="cuda")
    chunks = torch.zeros(1, dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError, match="nodes"):
        _lib.call("ibm_spread_noalloc", ctypes.byref(big.desc), ctypes.byref(sw.struct()), 0,
                  ptr(field), ptr(chunks), big.stream())
