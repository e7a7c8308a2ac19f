"""Launch-shape autotuner of the fused step kernel.

The fused step can run one node per thread, NZ consecutive z-nodes per
thread moved as 4 / 8 / 16-byte vectors (128 or 256 threads per block), or
as a persistent kernel that stages whole z-rows in shared memory with TMA
bulk copies.  The
best shape depends on the velocity set, the storage type and the row length,
so ``tune`` times every legal candidate with CUDA events on a scratch lattice
of the same velocity set, storage, faces and (ny, nz) -- with nx cut down so
the proxy still holds several times the L2 -- and caches the winner per
(q, storage, ny, nz, forced).  Tuning never touches the caller's populations.
"""
from __future__ import annotations

import torch

ROWS = -1   # whole z-rows staged in shared memory by TMA bulk copies
CANDIDATES = {
    32: [(1, 256), (2, 128), (2, 256), (4, 128), (4, 256), (ROWS, 256)],
    16: [(1, 256), (2, 128), (2, 256), (4, 128), (4, 256), (8, 128), (8, 256), (ROWS, 256)],
    64: [(1, 256), (2, 128), (2, 256)],
}
STORAGE_BITS = {"fp32": 32, "fp16s": 16, "bf16s": 16, "fp64": 64}
_CACHE = {}
PROXY_BYTES = 2 << 30          # populations of the proxy lattice (both buffers)


def shape_ok(nodes, pz, bits, nz=None):
    """Whether the fused step accepts `nodes` per thread on rows of pitch pz
    (nz: the row's node count when it differs from the pitch)."""
    nz = pz if nz is None else nz
    if nodes == 1:
        return True
    if nodes == ROWS:
        return bits != 64 and pz == nz and (nz * bits // 8) % 16 == 0 and nz >= 16
    if nodes * bits // 32 not in (1, 2, 4):
        return False
    if nodes == 2 and bits == 16 and pz % 2 == 1 and pz >= 3:
        return True                 # pairs within unpitched rows of odd length
    return pz % nodes == 0 and pz >= 2 * nodes


def default_shape(q, storage, pz, forced=False):
    """The launch shape lbm_flow_step uses when none is set (measured best on
    B200 at 512^3): node pairs with 128 threads where the rows allow them, 4
    nodes per thread for unforced D3Q13 / D3Q19 in 16-bit storage, else one
    node per thread."""
    bits = STORAGE_BITS[storage]
    want = 4 if (bits == 16 and q in (13, 19) and not forced) else 2
    for nodes in (want, 2):
        if pz % nodes == 0 and pz >= 2 * nodes:
            return (nodes, 128)
    return (1, 256)


# A candidate replaces the default shape only if its proxy timing is this much
# faster: short proxy timings scatter by a few percent, and the default is the
# measured best at full size.
MARGIN = 0.03


def _pick(timings, default):
    best = min(timings, key=timings.get)
    if default in timings and timings[default] <= timings[best] * (1.0 + MARGIN):
        return default
    return best


def tune(lat, force=None, iters=6, warmup=2, verbose=False):
    """Choose (nodes per thread, threads per block) for ``lat`` and store it
    in its descriptor.  Returns the choice and the timings in ms per step."""
    from .lattice import BYTES, Lattice

    bits = STORAGE_BITS[lat.storage]
    key = (lat.q, lat.storage, lat.shape[1], lat.shape[2], lat.pz, force is not None)
    if key in _CACHE:
        choice, timings = _CACHE[key]
        lat.set_launch_shape(*choice)
        return choice, timings
    nx, ny, nz = lat.shape
    per_x = 2 * lat.q * ny * nz * BYTES[lat.storage]
    px = max(4, min(nx, PROXY_BYTES // max(per_x, 1)))
    proxy = Lattice(lat.q, (px, ny, nz), lat.faces, lat.tau, storage=lat.storage,
                    face_uw=lat.face_uw, re_mu=lat.re_mu, device=lat.device,
                    pitch=lat.pz != nz)      # the lattice's own row layout
    proxy.init(None)
    timings = {}
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    for nodes, threads in CANDIDATES[bits]:
        if not shape_ok(nodes, proxy.pz, bits, nz):
            continue
        proxy.set_launch_shape(nodes, threads)
        for _ in range(warmup):
            proxy.step(force)
        start.record()
        for _ in range(iters):
            proxy.step(force)
        stop.record()
        stop.synchronize()
        timings[(nodes, threads)] = start.elapsed_time(stop) / iters
    proxy.release()
    del proxy
    choice = _pick(timings, default_shape(lat.q, lat.storage, lat.pz, force is not None))
    if verbose:
        for k, v in sorted(timings.items(), key=lambda kv: kv[1]):
            print("tune q=%d %s %dx%dx%d (proxy nx=%d): nodes=%d threads=%d  %.4f ms"
                  % (lat.q, lat.storage, nx, ny, nz, px, k[0], k[1], v))
    _CACHE[key] = (choice, timings)
    lat.set_launch_shape(*choice)
    return choice, timings


_CLASS_CACHE = {}
CLASS_PROXY_NODES = 96          # proxy lattice of a class: about 96^3 nodes


def class_key_of(q, storage, pz, forced):
    """Class of a lattice for the tuner: velocity set, storage, the vector
    widths its row pitch pz allows, forced or not."""
    return (int(q), storage, pz % 2 == 0 and pz >= 4, pz % 4 == 0 and pz >= 8,
            pz % 8 == 0 and pz >= 16, bool(forced))


def class_key(lat, forced):
    return class_key_of(lat.q, lat.storage, lat.pz, forced)


def tune_class_of(q, storage, nz, forced, device="cuda", iters=6, warmup=2):
    """Launch shape of the class (velocity set, storage, which vector widths
    rows of nz nodes allow, forced or not), tuned once per class on a ~96^3
    periodic proxy (forced: force fields in 5 % of the 32-node chunks, as
    spreading leaves them) and cached.  Meant for servers that see many
    lattice sizes: one short tuning per class instead of one per (ny, nz).
    Returns (nodes, threads)."""
    from .lattice import Lattice, make_force, tau_float32

    key = class_key_of(q, storage, nz, forced)
    if key in _CLASS_CACHE:
        return _CLASS_CACHE[key]
    _, _, even, by4, by8, _ = key
    pnz = 96 if by8 else 100 if by4 else 98 if even else 97
    n = CLASS_PROXY_NODES
    proxy = Lattice(int(q), (n, n, pnz), [11000] * 6, tau_float32(0.05), storage=storage,
                    device=device)
    proxy.init(None)
    force, keep = None, None
    if forced:
        # spread forces as IBM leaves them: fields in a few percent of the
        # 32-node chunks, none elsewhere (most threads run force-free)
        pn = proxy.n
        nch = (pn + 31) // 32
        dev = proxy.device
        g = torch.Generator(device="cpu").manual_seed(0)
        flags = (torch.rand(nch, generator=g) < 0.05).to(torch.uint8).to(dev)
        field = 1e-5 * torch.randn(pn, 3, device=dev)
        field *= flags.repeat_interleave(32)[:pn, None].to(field.dtype)
        keep = [field.reshape(-1), flags]
        force = make_force((0, 0, 0), (0, 0, 0), keep[0], keep[0], keep[1], keep[1])
    bits = STORAGE_BITS[storage]
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    timings = {}
    for nodes, threads in CANDIDATES[bits]:
        if nodes == ROWS or not shape_ok(nodes, proxy.pz, bits, pnz):
            continue
        proxy.set_launch_shape(nodes, threads)
        for _ in range(warmup):
            proxy.step(force)
        start.record()
        for _ in range(iters):
            proxy.step(force)
        stop.record()
        stop.synchronize()
        timings[(nodes, threads)] = start.elapsed_time(stop) / iters
    ppz = proxy.pz
    proxy.release()
    del proxy
    _CLASS_CACHE[key] = _pick(timings, default_shape(q, storage, ppz, forced))
    return _CLASS_CACHE[key]


def tune_class(lat, forced=False):
    """Set ``lat``'s launch shape to its class's tuned choice (tune_class_of)."""
    choice = tune_class_of(lat.q, lat.storage, lat.pz, forced, device=lat.device)
    lat.set_launch_shape(*choice)
    return choice


def clear_cache():
    _CACHE.clear()
    _CLASS_CACHE.clear()
