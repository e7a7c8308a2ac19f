"""Device state of one lattice on the fused path, over the C ABI.

A ``Lattice`` owns two population buffers in structure-of-arrays layout
``[q][x][y][z]`` and ping-pongs between
them: ``buf[cur]`` holds the post-collision populations the next step streams
from, ``buf[cur ^ 1]`` the ones the last step streamed from (kept for
observation).  fp32, fp16s and bf16s buffers hold the deviation d = f - w_i
of each population from its weight (float32, float16 scaled by 2^12,
bfloat16); fp64 buffers hold f.  Everything numeric runs in ``liblbm_b200.so``.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib
from ._lib import LbmForce, LbmLattice, LbmObserve, call, ptr

BC = {"PERIODICAL": 11000, "WALL": 1200, "WALL_WITH_SPEED": 1201, "NON_EQUILIBRIUM": 1400}
STORAGE_DTYPE = {"fp32": torch.float32, "fp16s": torch.float16, "bf16s": torch.bfloat16,
                 "fp64": torch.float64}
BYTES = {"fp32": 4, "fp16s": 2, "bf16s": 2, "fp64": 8}
# fp16s buffers hold (f - w) * FP16_SCALE (kept out of float16's subnormals)
FP16_SCALE = 4096.0
# elements of the widest vector (16 bytes) the step moves per thread: the
# population rows are pitched to a multiple of it
VECTOR_ELEMS = {"fp32": 4, "fp16s": 8, "bf16s": 8, "fp64": 2}


# 16-bit lattices of at least this many nodes pitch rows of odd length
PITCH_MIN_NODES = 1 << 24


def default_pitch(shape, storage):
    """Whether a lattice pitches its population rows unless told otherwise:
    16-bit storage, rows of odd length, at least 2^24 nodes.  Measured on
    B200 (D3Q19 fp16s): pitched rows let node pairs run and win 9 % at 257^3
    (322 against 351 us per step on dense rows); on the walled 161x65x65
    and 257x129x129 lattices one node per thread on dense rows wins (23.0
    against 27.0 us, 162.6 against 173.2 us); in FP32 dense rows win
    (257^3: 435 us dense, 448 us pitched)."""
    shape = tuple(int(s) for s in shape)
    return (BYTES[storage] == 2 and shape[2] % 2 == 1
            and shape[0] * shape[1] * shape[2] >= PITCH_MIN_NODES)


def row_pitch(nz, storage):
    """Row pitch of the population buffers: nz rounded up to the widest vector,
    so that rows of any length (the reference's size + 1 nodes are odd for
    even sizes) run the vectorised step."""
    w = VECTOR_ELEMS[storage]
    return -(-int(nz) // w) * w


# arithmetic type of a storage: what its fields, face densities, force fields
# and observation buffers hold
REAL_DTYPE = {"fp32": torch.float32, "fp16s": torch.float32, "bf16s": torch.float32,
              "fp64": torch.float64}


def cs2_float32():
    """cs = float32(sqrt(1/3)) squared in float32 (flow/base.py:37-39)."""
    cs = np.float32(math.sqrt(1.0 / 3))
    return float(np.float32(cs * cs))


def tau_float32(mu):
    """tau = float32(3 mu + 0.5) (flow/d3/base.py:96)."""
    return float(np.float32(3 * float(mu) + 0.5))


def duct_profile(a, b, n_max=100):
    """Inlet profile of the NON_EQUILIBRIUM face: the reference's ``cul_u``
    series (flow/d3/base.py:10-37) on the ``init_u`` grid, each value rounded
    to 6 decimals; float64 [a, b]."""
    y = np.linspace(-(a - 1) / 2, (a - 1) / 2, a)
    z = np.linspace(-(b - 1) / 2, (b - 1) / 2, b)
    ha, hb = a / 2.0, b / 2.0
    n = np.arange(n_max)
    nt = (2 * n + 1)[None, None, :]
    base = 32 * (-1.0) ** (n + 1) / ((2 * n + 1) ** 3 * np.pi ** 3)
    Y = y[:, None, None]
    Z = z[None, :, None]
    terms = base * np.cos(nt * np.pi * Y / (2 * ha)) * (
        np.cosh(nt * np.pi * Z / (2 * ha)) / np.cosh(nt * np.pi * hb / (2 * ha)))
    val = 1 - (Y[..., 0] / ha) ** 2 + terms.sum(-1)
    return np.round(val, 6)


class Lattice:
    """One lattice: descriptor, population buffers, face-density planes."""

    def __init__(self, q, shape, faces, tau, storage="fp32", face_uw=None, re_mu=0.0,
                 device="cuda", allocate=True, pitch=None):
        if storage not in STORAGE_DTYPE:
            raise ValueError("unknown storage %r (fp32, fp16s, bf16s)" % (storage,))
        self.q = int(q)
        self.shape = tuple(int(s) for s in shape)
        self.n = self.shape[0] * self.shape[1] * self.shape[2]
        # population rows pitched to the vector width (pitch=False: dense
        # rows; None: default_pitch)
        if pitch is None:
            pitch = default_pitch(self.shape, storage)
        self.pz = row_pitch(self.shape[2], storage) if pitch else self.shape[2]
        self.np = self.shape[0] * self.shape[1] * self.pz
        self.storage = storage
        self.device = torch.device(device)
        self.faces = [int(c) for c in faces]
        self.face_uw = [tuple(float(v) for v in (face_uw[i] if face_uw else (0, 0, 0)))
                        for i in range(6)]
        self.tau = float(tau)
        self.re_mu = float(np.float32(re_mu))
        self._profile = None
        if self.faces[0] == BC["NON_EQUILIBRIUM"]:
            prof = duct_profile(self.shape[1], self.shape[2])
            self._profile = torch.tensor(prof.reshape(-1), dtype=torch.float64, device=self.device)
        self.desc = self._make_desc(storage)
        self.desc.pz = self.pz
        self.desc_fp32 = self._make_desc("fp32")     # dense: the single-function calls
        call("lbm_lattice_check", ctypes_ref(self.desc))
        self.needs_face_rho = any(c in (BC["WALL_WITH_SPEED"], BC["NON_EQUILIBRIUM"]) for c in self.faces)
        self.fused = BC["NON_EQUILIBRIUM"] not in self.faces
        self.buf = [None, None]
        self.face_rho = [None, None]
        self.cur = 0
        self.status = None
        if allocate:
            self.allocate()

    def _make_desc(self, storage):
        d = LbmLattice()
        d.q = self.q
        d.nx, d.ny, d.nz = self.shape
        for i in range(6):
            d.face[i] = self.faces[i]
            for k in range(3):
                d.face_uw[i][k] = self.face_uw[i][k]
        d.tau = self.tau
        d.cs2 = cs2_float32()
        d.storage = _lib.STORAGE[storage]
        d.re_mu = self.re_mu
        d.neq_profile = None if self._profile is None else self._profile.data_ptr()
        return d

    # -- memory ------------------------------------------------------------
    @staticmethod
    def bytes_needed(q, shape, storage="fp32", pitch=None):
        if pitch is None:
            pitch = default_pitch(shape, storage)
        pz = row_pitch(shape[2], storage) if pitch else int(shape[2])
        n = int(shape[0]) * int(shape[1]) * pz
        planes = 2 * (shape[1] * shape[2] + shape[0] * shape[2] + shape[0] * shape[1])
        return 2 * q * n * BYTES[storage] + 2 * REAL_DTYPE[storage].itemsize * planes

    def allocate(self):
        dt = STORAGE_DTYPE[self.storage]
        for i in range(2):
            if self.buf[i] is None:
                self.buf[i] = torch.empty(self.q * self.np, dtype=dt, device=self.device)
        if self.needs_face_rho and self.face_rho[0] is None:
            nplanes = _lib.load().lbm_face_plane_floats(ctypes_ref(self.desc))
            self.face_rho = [torch.zeros(nplanes, dtype=REAL_DTYPE[self.storage],
                                         device=self.device) for _ in range(2)]
        if self.status is None:
            self.status = torch.zeros(1, dtype=torch.int32, device=self.device)

    def release(self):
        self.buf = [None, None]
        self.face_rho = [None, None]

    # -- steps -------------------------------------------------------------
    def stream(self):
        return _lib.stream_of(torch, self.device)

    @property
    def real_dtype(self):
        return REAL_DTYPE[self.storage]

    def init(self, f0=None):
        """Post-collision populations of step 1 from f0 (SoA in the storage's
        arithmetic type: float64 for fp64, float32 otherwise) or rho*w."""
        if f0 is not None and f0.dtype != self.real_dtype:
            raise TypeError("initial field of a %s lattice must be %s" % (self.storage,
                                                                          self.real_dtype))
        call("lbm_flow_init", ctypes_ref(self.desc), ptr(f0), ptr(self.buf[self.cur]),
             ptr(self.face_rho[self.cur]), self.stream())

    def load_post_collision_fp32(self, a):
        """Adopt float32 SoA post-collision populations (dense [q][x][y][z];
        storage conversion and row pitch on the device)."""
        X, Y, Z = self.shape
        dst = self.buf[self.cur].view(self.q, X * Y, self.pz)[:, :, :Z]
        src = a.reshape(self.q, X * Y, Z)
        if self.storage == "fp64":
            dst.copy_(src)
        else:
            w = weights_tensor(self.q, self.device)
            d = src - w[:, None, None]
            if self.storage == "fp16s":
                d = d * FP16_SCALE
            dst.copy_(d.to(STORAGE_DTYPE[self.storage]))

    def step(self, force=None, obs=None):
        nxt = self.cur ^ 1
        call("lbm_flow_step", ctypes_ref(self.desc), ptr(self.buf[self.cur]), ptr(self.buf[nxt]),
             None if force is None else ctypes_ref(force), ptr(self.face_rho[self.cur]),
             ptr(self.face_rho[nxt]), None if obs is None else ctypes_ref(obs),
             ptr(self.status), self.stream())
        self.cur = nxt

    def observe(self, force, f=None, rho=None, u=None):
        """Reference state at the end of the last step (f after cul_equ2,
        rou / u after the second update_u_rou), recomputed from the buffer the
        last step streamed from."""
        prev = self.cur ^ 1
        obs = LbmObserve(ptr(f), ptr(rho), ptr(u))
        call("lbm_flow_step", ctypes_ref(self.desc), ptr(self.buf[prev]), None,
             None if force is None else ctypes_ref(force), ptr(self.face_rho[prev]), None,
             ctypes_ref(obs), None, self.stream())

    def stats(self, force, out=None):
        """min, mean, max of f, u, rho at the end of the last step (9 float64
        values on the device), from the buffer the last step streamed from."""
        prev = self.cur ^ 1
        if out is None:
            out = torch.empty(9, dtype=torch.float64, device=self.device)
        call("lbm_flow_stats", ctypes_ref(self.desc), ptr(self.buf[prev]),
             None if force is None else ctypes_ref(force), ptr(self.face_rho[prev]), ptr(out),
             ptr(self.status), self.stream())
        return out

    def set_launch_shape(self, nodes=0, threads=0):
        """Launch shape of the fused step (see funlbm_b200.tune)."""
        for d in (self.desc,):
            d.step_nodes = int(nodes)
            d.step_threads = int(threads)

    def tune(self, force=None, verbose=False):
        from .tune import tune

        return tune(self, force=force, verbose=verbose)

    def read_status(self, reset=True):
        v = int(self.status.item())
        if reset:
            self.status.zero_()
        return v


def make_force(old_uniform=(0, 0, 0), new_uniform=(0, 0, 0), old_field=None, new_field=None,
               old_chunks=None, new_chunks=None):
    f = LbmForce()
    for k in range(3):
        f.old_uniform[k] = float(old_uniform[k])
        f.new_uniform[k] = float(new_uniform[k])
    f.old_field = None if old_field is None else old_field.data_ptr()
    f.new_field = None if new_field is None else new_field.data_ptr()
    f.old_chunks = None if old_chunks is None else old_chunks.data_ptr()
    f.new_chunks = None if new_chunks is None else new_chunks.data_ptr()
    return f


def ctypes_ref(s):
    import ctypes

    return ctypes.byref(s)


_WCACHE = {}


def velocity_set(q):
    """(e [q,3] int, w [q] float64, rev [q]) in the reference's direction order
    (flow/d3/d3q13.py, d3q15.py, d3q19.py, d3q27.py)."""
    from .flow import VELOCITY_SETS

    e = np.array(VELOCITY_SETS[q][0], dtype=np.int64)
    w = np.array(VELOCITY_SETS[q][1], dtype=np.float64)
    lookup = {tuple(v): i for i, v in enumerate(e.tolist())}
    rev = np.array([lookup[tuple((-v).tolist())] for v in e], dtype=np.int64)
    return e, w, rev


def weights_tensor(q, device):
    key = (q, str(device))
    if key not in _WCACHE:
        _WCACHE[key] = torch.tensor(velocity_set(q)[1], dtype=torch.float32, device=device)
    return _WCACHE[key]
