"""Rigid particles with the reference's API (funlbm ``particle/``).

``CoordConfig``, ``Coordinate``, ``ParticleConfig``, ``Particle``, ``Sphere``,
``Ellipsoid``, ``ParticleSwarm``, ``create_particle``,
``create_particle_swarm``.  Marker generation and mass properties run once on
the host at init (as in the reference); afterwards the whole swarm lives on
the device as concatenated arrays in the reference's (particle, marker)
order, and every per-step update is a kernel of liblbm_b200.so.  Each
``Particle``'s attributes (``cx, cu, cw, cF, cT, lx, lF, lu, lm, lrou``,
``coord.angle``) are views into those arrays.
"""
from __future__ import annotations

import ctypes
import math
from typing import List

import numpy as np
import torch

from . import _lib
from ._lib import LbmParticles, call
from .config import BaseConfig, deep_get


def _device(device):
    from .flow import _device as fd

    return fd(device)


# ---------------------------------------------------------------------------
# Marker generation (particle/base/ellipsoid.py:10-95), vectorised
# ---------------------------------------------------------------------------
_CORNERS = [(a, b, c) for a in (0, 1) for b in (0, 1) for c in (0, 1)]
_PAIRS = [(i, j) for i in range(8) for j in range(i + 1, 8)]


def generate_uniform_points_on_ellipsoid(xl, yl, zl, xr, yr, zr, cul_value=None, dx=0.5,
                                         semi_axes=None, *args, **kwargs):
    """Surface markers of an ellipsoid by the reference's cube-crossing rule.

    The box [xl, xr) x [yl, yr) x [zl, zr) is cut into cubes of edge dx; every
    cube whose corners lie on both sides of the surface yields the centroid of
    the surface crossings on all of its corner pairs of opposite sides (when
    there are at least three).  ``semi_axes`` = (a, b, c) selects the
    ellipsoid x^2/a^2 + y^2/b^2 + z^2/c^2 = 1, whose crossing on a segment is
    the root of a quadratic (solved in closed form; the reference iterates
    with fsolve to the same root).  ``cul_value`` (the reference's implicit
    function) is accepted for signature compatibility when semi_axes is given.
    """
    if semi_axes is None:
        raise ValueError("semi_axes=(a, b, c) is required")
    a, b, c = (float(v) for v in semi_axes)
    xs = np.arange(xl, xr, dx)
    ys = np.arange(yl, yr, dx)
    zs = np.arange(zl, zr, dx)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    # term by term as the reference writes it, so that corners exactly on the
    # surface classify identically
    inside = (X ** 2 / a ** 2 + Y ** 2 / b ** 2 + Z ** 2 / c ** 2 - 1) < 0
    nx, ny, nz = len(xs) - 1, len(ys) - 1, len(zs) - 1
    if min(nx, ny, nz) <= 0:
        return np.zeros((0, 3))
    corner_in = np.stack([inside[i:i + nx, j:j + ny, k:k + nz] for (i, j, k) in _CORNERS], -1)
    mixed = corner_in.any(-1) & ~corner_in.all(-1)
    ci, cj, ck = np.nonzero(mixed)                      # C order = the reference's loop order
    if ci.size == 0:
        return np.zeros((0, 3))
    cin = corner_in[ci, cj, ck]                          # [M, 8]
    verts = np.stack([np.stack([xs[ci + i], ys[cj + j], zs[ck + k]], -1) for (i, j, k) in _CORNERS], 1)
    inv = np.array([1.0 / a ** 2, 1.0 / b ** 2, 1.0 / c ** 2])
    p1 = verts[:, [p[0] for p in _PAIRS]]                # [M, 28, 3]
    p2 = verts[:, [p[1] for p in _PAIRS]]
    d = p2 - p1
    A = (d * d * inv).sum(-1)
    B = 2 * (p1 * d * inv).sum(-1)
    C = (p1 * p1 * inv).sum(-1) - 1
    sq = np.sqrt(np.maximum(B * B - 4 * A * C, 0.0))
    with np.errstate(divide="ignore", invalid="ignore"):
        r1 = (-B - sq) / (2 * A)
        r2 = (-B + sq) / (2 * A)
    t = np.where(np.abs(r1 - 0.5) <= np.abs(r2 - 0.5), r1, r2)
    cross = p1 + t[..., None] * d                        # [M, 28, 3]
    differs = cin[:, [p[0] for p in _PAIRS]] != cin[:, [p[1] for p in _PAIRS]]
    counts = differs.sum(-1)
    out = []
    for m in np.nonzero(counts >= 3)[0]:
        out.append(np.mean(cross[m][differs[m]], axis=0))
    return np.array(out) if out else np.zeros((0, 3))


# ---------------------------------------------------------------------------
# Coordinates (particle/coord.py)
# ---------------------------------------------------------------------------
class CoordConfig(BaseConfig):
    """particle/coord.py:13-43; missing keys fall back to the defaults."""

    def __init__(self, alpha: float = np.pi / 2, beta: float = 0, gamma: float = 0, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.center = [0, 0, 0]
        self.alpha, self.beta, self.gamma = alpha, beta, gamma

    def _from_json(self, config_json, *args, **kwargs):
        self.center = deep_get(config_json, "center") or self.center
        self.alpha = deep_get(config_json, "alpha") or self.alpha
        self.beta = deep_get(config_json, "beta") or self.beta
        self.gamma = deep_get(config_json, "gamma") or self.gamma


def rotvec_matrix(v):
    """Rotation matrix (float64) of a rotation vector through the unit quaternion."""
    v = np.asarray(v, np.float64)
    th = float(np.sqrt(v @ v))
    if th <= 1e-3:
        t2 = th * th
        s = 0.5 - t2 / 48 + t2 * t2 / 3840
    else:
        s = math.sin(th / 2) / th
    x, y, z = s * v
    w = math.cos(th / 2)
    n = math.sqrt(x * x + y * y + z * z + w * w)
    x, y, z, w = x / n, y / n, z / n, w / n
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


class Coordinate:
    """Body frame of a particle (particle/coord.py:46-120).  ``angle`` is the
    accumulated rotation vector; ``center`` the centre of mass."""

    def __init__(self, config: CoordConfig = None, device="cuda", dtype=torch.float32, *args,
                 **kwargs):
        config = config or CoordConfig()
        self.device = _device(device)
        self._center = torch.tensor(config.center, device=self.device, dtype=dtype)
        self._angle = torch.tensor([config.alpha, config.beta, config.gamma], device=self.device,
                                   dtype=dtype)

    @property
    def center(self):
        return self._center

    @center.setter
    def center(self, v):
        self._center.copy_(torch.as_tensor(v, dtype=self._center.dtype))

    @property
    def angle(self):
        return self._angle

    @angle.setter
    def angle(self, v):
        self._angle.copy_(torch.as_tensor(v, dtype=self._angle.dtype))

    @property
    def rotation(self):
        return rotvec_matrix(self._angle.detach().cpu().numpy())

    def cul_point(self, points):
        """Rotate body-frame points by ``angle`` and translate by ``center``."""
        pts = np.asarray(points.detach().cpu().numpy() if isinstance(points, torch.Tensor) else points,
                         np.float64)
        rot = pts @ self.rotation.T
        return torch.tensor(rot, device=self.device, dtype=self._center.dtype) + self._center

    def update(self, center, w):
        self.center = center
        self.angle = self._angle + w

    def to_str(self):
        return ("center=" + ",".join("%.6f" % v for v in self._center.tolist()) + "\tangle="
                + ",".join("%.6f" % v for v in self._angle.tolist()))

    def to_json(self):
        return {"center": self._center.tolist(), "angle": self._angle.tolist()}


# ---------------------------------------------------------------------------
# Particles (particle/base/base.py, sphere.py, ellipsoid.py)
# ---------------------------------------------------------------------------
class ParticleConfig(BaseConfig):
    """particle/base/base.py:11-19 (a missing ``coord`` block means defaults;
    the reference raises TypeError there)."""

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.coord_config = CoordConfig()
        self.type = "ellipsoid"

    def _from_json(self, config_json, *args, **kwargs):
        self.coord_config.from_json(deep_get(config_json, "coord") or {})
        self.type = deep_get(config_json, "type") or self.type


_STATE = ("cx", "cu", "cw", "cF", "cT")
_MARKER = ("lx", "lF", "lu", "lm", "lrou", "_lagrange")


class Particle:
    """Rigid particle (particle/base/base.py:22-214).  Before the swarm packs
    it the state lives in its own tensors; afterwards in the swarm arrays.
    ``dtype`` is float32 (the reference's) or float64 (particles of an FP64
    lattice)."""

    def __init__(self, config: ParticleConfig = None, device="cuda", dtype=torch.float32, *args,
                 **kwargs):
        self.device = _device(device)
        self.dtype = dtype
        self.config = config or ParticleConfig()
        self.coord = Coordinate(config=self.config.coord_config, device=self.device, dtype=dtype)
        self.mass = None
        self.area = None
        self.I = None
        self.rou = None
        self._t = {
            "cx": torch.tensor(self.config.coord_config.center, device=self.device, dtype=dtype),
            "cu": torch.zeros(3, device=self.device, dtype=dtype),
            "cw": torch.zeros(3, device=self.device, dtype=dtype),
            "cF": torch.zeros(3, device=self.device, dtype=dtype),
            "cT": torch.zeros(3, device=self.device, dtype=dtype),
        }
        for k in _MARKER:
            self._t[k] = torch.zeros([0], device=self.device, dtype=dtype)
        self._swarm = None
        self._index = None

    def _init(self, dx=1, *args, **kwargs):
        raise NotImplementedError("not implemented")

    def init(self, *args, **kwargs):
        """particle/base/base.py:108-118: markers, mass properties; markers sit
        at the origin until the first update (the reference's lx = zeros)."""
        self.rou = float(self.config.get("rou", 1.0))
        self._init(*args, **kwargs)
        n = self._t["_lagrange"].shape[0]
        dt = self.dtype
        self._t["lx"] = torch.zeros((n, 3), device=self.device, dtype=dt)
        self._t["lF"] = torch.zeros((n, 3), device=self.device, dtype=dt)
        self._t["lu"] = torch.zeros((n, 3), device=self.device, dtype=dt)
        # lm = area / N as a tensor division, like torch.full((N, 1), area / N)
        self._t["lm"] = ((self.area / n).reshape(1, 1).expand(n, 1).contiguous() if n
                         else torch.zeros((0, 1), device=self.device, dtype=dt))
        self._t["lrou"] = torch.zeros((n, 1), device=self.device, dtype=dt)

    # attribute views ---------------------------------------------------------
    def _view(self, key):
        return self._t[key]

    def __getattr__(self, key):
        if key in _STATE or key in _MARKER:
            return self.__dict__["_t"][key]
        raise AttributeError(key)

    def __setattr__(self, key, value):
        if key in _STATE or key in _MARKER:
            t = self.__dict__["_t"][key]
            v = torch.as_tensor(value, dtype=t.dtype, device=t.device)
            if t.numel() == v.numel() and t.numel() > 0:
                t.copy_(v.reshape(t.shape))
            else:
                self.__dict__["_t"][key] = v.clone()
            sw = self.__dict__.get("_swarm")
            if key == "lx" and sw is not None:
                sw.ext_valid = False
            return
        object.__setattr__(self, key, value)

    # per-particle reference methods ------------------------------------------
    def update_from_lar(self, dt: float, gl: float = 9.8, rouf: float = 1.0) -> None:
        """particle/base/base.py:120-151 (float64 sums over markers)."""
        if dt <= 0:
            raise ValueError("Time step must be positive")
        if rouf <= 0:
            raise ValueError("Fluid density must be positive")
        self._require_swarm()
        sw = self._swarm
        call("rigid_wall_and_update", None, ctypes.byref(sw.single(self._index)),
             _lib.RIGID_UPDATE, float(dt), 1.0, float(gl), float(rouf), sw.stream())

    def update(self, dt=1.0):
        """particle/base/base.py:153-156: angle += cw; lx = R(angle) X0 + cx."""
        self._require_swarm()
        sw = self._swarm
        call("rigid_update_markers", ctypes.byref(sw.single(self._index)), sw.stream())
        sw.ext_valid = False

    def _require_swarm(self):
        if self._swarm is None:
            ParticleSwarm.adopt([self], self.device)

    def to_str(self, step=0, *args, **kwargs):
        def fmt(t):
            return ",".join("%.6f" % v for v in t.tolist())

        lf = self.lF
        res = "m=%.2f" % float(self.mass)
        res += "\tcu=" + fmt(self.cu) + "\tcx=" + fmt(self.cx) + "\tcf=" + fmt(self.cF)
        res += "\tlF=" + ",".join("%.6f" % float(v) for v in (lf.min(), lf.mean(), lf.max()))
        res += "\tcw=" + fmt(self.cw) + "\tr=" + self.coord.to_str()
        return res

    def to_json(self, step=0, *args, **kwargs):
        lf = self.lF
        return {"m": float(self.mass), "cu": self.cu.tolist(), "cx": self.cx.tolist(),
                "cf": self.cF.tolist(),
                "lF": [float(lf.min()), float(lf.mean()), float(lf.max())],
                "cw": self.cw.tolist(), "coord": self.coord.to_json()}

    def dump_checkpoint(self, group=None, *args, **kwargs):
        if group is None:
            return
        for k in ("cu", "cx", "cF", "cw", "lx", "lF", "lu", "lrou"):
            group.create_dataset(k, data=getattr(self, k).cpu().numpy(), compression="gzip",
                                 compression_opts=9)
        group.create_dataset("angle", data=self.coord.angle.cpu().numpy())

    def load_checkpoint(self, group=None, *args, **kwargs):
        if group is None:
            return
        for k in ("cu", "cx", "cF", "cw", "lx", "lF", "lu", "lrou"):
            setattr(self, k, np.asarray(group.get(k)[:]))
        if group.get("angle") is not None:
            self.coord.angle = torch.tensor(np.asarray(group.get("angle")[:]))


_MARKER_CACHE = {}


def _markers_tensor(ra, rb, rc, dx, device, dtype=torch.float32):
    """Body-frame markers of an ellipsoid (a sphere when ra = rb = rc); the
    generator is deterministic, so each shape is computed once per process."""
    key = (float(ra), float(rb), float(rc), float(dx))
    if key not in _MARKER_CACHE:
        _MARKER_CACHE[key] = generate_uniform_points_on_ellipsoid(
            -ra - 2 * dx, -rb - 2 * dx, -rc - 2 * dx, ra + 2 * dx, rb + 2 * dx, rc + 2 * dx,
            dx=dx, semi_axes=(ra, rb, rc))
    pts = _MARKER_CACHE[key]
    return torch.tensor(pts, device=device, dtype=dtype).reshape(-1, 3)


class Sphere(Particle):
    """particle/base/sphere.py:10-53"""

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.r = self.config.get("r") or 10

    def _init(self, dx=1, *args, **kwargs):
        r = self.r
        dt = self.dtype
        self._t["_lagrange"] = _markers_tensor(r, r, r, dx, self.device, dt)
        self.mass = torch.tensor(4.0 / 3.0 * math.pi * r * r * r, device=self.device, dtype=dt)
        self.area = torch.tensor(4.0 * math.pi * r * r, device=self.device, dtype=dt)
        self.I = torch.tensor(np.array([r * r, r * r, r * r]) * self.mass.cpu().numpy() / 5.0,
                              device=self.device, dtype=dt)


class Ellipsoid(Particle):
    """particle/base/ellipsoid.py:98-143"""

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.ra = self.config.get("a") or 10
        self.rb = self.config.get("b") or 10
        self.rc = self.config.get("c") or 10

    def _init(self, dx=1, *args, **kwargs):
        a, b, c = self.ra, self.rb, self.rc
        dt = self.dtype
        self._t["_lagrange"] = _markers_tensor(a, b, c, dx, self.device, dt)
        self.mass = torch.tensor(4.0 / 3.0 * math.pi * a * b * c, device=self.device, dtype=dt)
        self.area = torch.tensor(4.0 / 3.0 * math.pi * math.pow(a * b * c, 2.0 / 3.0),
                                 device=self.device, dtype=dt)
        self.I = torch.tensor(np.array([b * c, a * c, a * b]) * self.mass.cpu().numpy() / 5.0,
                              device=self.device, dtype=dt)


def create_particle(config: ParticleConfig, device="cuda", dtype=torch.float32) -> Particle:
    """particle/base/__init__.py:8-12"""
    if config.type == "ellipsoid":
        return Ellipsoid(config=config, device=device, dtype=dtype)
    return Sphere(config=config, device=device, dtype=dtype)


class ParticleSwarm:
    """particle/swarm.py:12-41, with the device arrays of all particles."""

    def __init__(self, configs: List[ParticleConfig] = (), device="cuda", dtype=torch.float32):
        self.device = _device(device)
        self.dtype = dtype
        self.particles: List[Particle] = [create_particle(c, device=self.device, dtype=dtype)
                                          for c in configs]
        self._packed = False

    @classmethod
    def adopt(cls, particles, device):
        dtype = particles[0].dtype if particles else torch.float32
        sw = cls((), device, dtype=dtype)
        sw.particles = list(particles)
        sw.pack()
        return sw

    def init(self, *args, **kwargs):
        for p in self.particles:
            p.init(*args, **kwargs)
        self.pack()

    @property
    def n_markers(self):
        return int(self._offsets_host[-1]) if self._packed else 0

    def pack(self):
        """Concatenate the particles' state into device arrays and rebind
        every particle attribute as a view of them."""
        dev = self.device
        ps = self.particles
        counts = [int(p._t["_lagrange"].shape[0]) for p in ps]
        offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        self._offsets_host = offs
        self.offsets = torch.tensor(offs, dtype=torch.int32, device=dev)
        self.owner = torch.tensor(np.repeat(np.arange(len(ps)), counts).astype(np.int32), device=dev)
        M = int(offs[-1])
        P = len(ps)

        dt = self.dtype

        def cat_markers(key, width):
            if M == 0:
                return torch.zeros((0, width), device=dev, dtype=dt)
            return torch.cat([p._t[key].reshape(-1, width).to(dt) for p in ps]).contiguous()

        self.lagrange = cat_markers("_lagrange", 3)
        self.lx = cat_markers("lx", 3)
        self.lF = cat_markers("lF", 3)
        self.lu = cat_markers("lu", 3)
        self.lm = cat_markers("lm", 1)
        self.lrou = cat_markers("lrou", 1)

        def stack(key):
            return (torch.stack([p._t[key].to(dt) for p in ps]).contiguous() if P
                    else torch.zeros((0, 3), device=dev, dtype=dt))

        self.cx, self.cu, self.cw, self.cF, self.cT = (stack(k) for k in _STATE)
        self.angle = (torch.stack([p.coord.angle.to(dt) for p in ps]).contiguous() if P
                      else torch.zeros((0, 3), device=dev, dtype=dt))
        self.mass = torch.tensor([float(p.mass) for p in ps], dtype=dt, device=dev)
        self.inertia = (torch.stack([p.I.to(dt) for p in ps]).contiguous() if P
                        else torch.zeros((0, 3), device=dev, dtype=dt))
        self.rou = torch.tensor([float(p.rou) for p in ps], dtype=dt, device=dev)
        for i, p in enumerate(ps):
            a, b = int(offs[i]), int(offs[i + 1])
            for key, arr in (("_lagrange", self.lagrange), ("lx", self.lx), ("lF", self.lF),
                             ("lu", self.lu), ("lm", self.lm), ("lrou", self.lrou)):
                p._t[key] = arr[a:b]
            for key in _STATE:
                p._t[key] = getattr(self, key)[i]
            p.coord._angle = self.angle[i]
            p.coord._center = self.cx[i]
            p._swarm = self
            p._index = i
        # the wall spring's six extreme markers of each particle (kept by
        # rigid_step; recomputed by rigid_extremes when positions changed
        # any other way)
        self.extreme = torch.zeros((max(P, 1), 6), dtype=torch.int32, device=dev)
        self.ext_valid = False
        self._singles = {}
        self._struct = self._make_struct(0, P, offs, self.owner, self.offsets)
        self._packed = True

    def _make_struct(self, p0, p1, offs, owner, offsets):
        s = LbmParticles()
        m0 = int(offs[p0])
        s.n_particles = p1 - p0
        s.n_markers = int(offs[p1]) - m0

        def at(t, row):
            return None if t.numel() == 0 else t.data_ptr() + row * t.stride(0) * t.element_size()

        s.marker_offset = offsets.data_ptr()
        s.marker_owner = owner.data_ptr()
        s.lagrange = at(self.lagrange, m0)
        s.lx = at(self.lx, m0)
        s.lu = at(self.lu, m0)
        s.lF = at(self.lF, m0)
        s.lrou = at(self.lrou, m0)
        s.lm = at(self.lm, m0)
        for key in _STATE + ("angle",):
            setattr(s, key, at(getattr(self, key), p0))
        s.mass = at(self.mass, p0)
        s.inertia = at(self.inertia, p0)
        s.rou = at(self.rou, p0)
        s.fp64 = 1 if self.dtype == torch.float64 else 0
        s.extreme = self.extreme.data_ptr() + p0 * 6 * 4
        return s

    def struct(self):
        if not self._packed:
            self.pack()
        return self._struct

    def single(self, i):
        """Descriptor of particle i alone (for the per-particle methods)."""
        if i not in self._singles:
            offs = self._offsets_host
            n = int(offs[i + 1] - offs[i])
            offsets = torch.tensor([0, n], dtype=torch.int32, device=self.device)
            owner = torch.zeros(max(n, 1), dtype=torch.int32, device=self.device)
            self._singles[i] = (self._make_struct(i, i + 1, offs, owner, offsets), offsets, owner)
        return self._singles[i][0]

    def stream(self):
        return _lib.stream_of(torch, self.device)

    def update(self, *args, **kwargs):
        """particle/swarm.py:22-24 for all particles in one launch."""
        if not self.particles:
            return
        call("rigid_update_markers", ctypes.byref(self.struct()), self.stream())
        self.ext_valid = False

    def ensure_extremes(self):
        """Make `extreme` hold the extreme markers of the current positions."""
        if self.particles and not self.ext_valid:
            call("rigid_extremes", ctypes.byref(self.struct()), self.stream())
            self.ext_valid = True

    def save_particle(self):
        pass

    def dump_checkpoint(self, group=None, *args, **kwargs):
        for i, particle in enumerate(self.particles):
            particle.dump_checkpoint(group.create_group("particle_%06d" % i), *args, **kwargs)

    def load_checkpoint(self, group=None, *args, **kwargs):
        for i, particle in enumerate(self.particles):
            particle.load_checkpoint(group.get("particle_%06d" % i), *args, **kwargs)
        self.ext_valid = False


def create_particle_swarm(configs: List[ParticleConfig] = (), device="cuda", dtype=torch.float32,
                          *args, **kwargs):
    return ParticleSwarm(configs=configs, device=device, dtype=dtype)
