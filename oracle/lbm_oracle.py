"""Oracle: numpy restatement of funlbm's per-step LBM hot path.

TEST INFRASTRUCTURE ONLY -- the checker, never the product.  Imported only by
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``.

Each function restates one reference function (cited as ``file:line`` inside
the funlbm source tree ``src/funlbm/``) in plain numpy, with the reference's
quirks kept (grid of size+1 nodes, velocity zeroed on all six planes, periodic
faces without transverse shift, last-override-wins streaming, scalar IBM
interpolation, last-writer-wins spreading, 0.1 torque factor, ...).

``dtype=np.float32`` follows the reference's float32 arithmetic step by step;
``dtype=np.float64`` gives the FP64 comparison run used for the shifted-storage
error figures.

Parity pin: the float32 mode is checked against golden vectors written by the
reference itself (``tests/golden/make_golden.py`` -> ``tests/golden/*.npz``).

Two reference paths crash as shipped (WALL_WITH_SPEED reads ``uw`` through a
``x or default`` lookup; NON_EQUILIBRIUM passes a tensor to ``torch.from_numpy``).
The oracle implements them with the minimal fix (``uw`` as a float vector, the
inlet ``u_max`` as a Python float); the golden script applies the same two
patches to the reference before recording them.
"""
from __future__ import annotations

import math

import numpy as np

# --------------------------------------------------------------------------
# Velocity sets (flow/d3/d3q13.py:7-44, d3q15.py:7-48, d3q19.py:7-60,
# d3q27.py:7-77).  Direction order is the reference's: the opposite-direction
# table and the [X, Y, Z, Q] population layout depend on it.
# --------------------------------------------------------------------------
_E = {
    13: [(0, 0, 0), (1, 1, 0), (1, -1, 0), (1, 0, 1), (1, 0, -1), (0, 1, 1), (0, 1, -1),
         (-1, -1, 0), (-1, 1, 0), (-1, 0, -1), (-1, 0, 1), (0, -1, -1), (0, -1, 1)],
    15: [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
         (1, 1, 1), (-1, 1, 1), (1, -1, 1), (-1, -1, 1), (1, 1, -1), (-1, 1, -1),
         (1, -1, -1), (-1, -1, -1)],
    19: [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
         (1, 1, 0), (-1, 1, 0), (1, -1, 0), (-1, -1, 0), (0, 1, 1), (0, -1, 1), (0, 1, -1),
         (0, -1, -1), (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1)],
    27: [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
         (1, 1, 0), (-1, 1, 0), (1, -1, 0), (-1, -1, 0), (0, 1, 1), (0, -1, 1), (0, 1, -1),
         (0, -1, -1), (1, 0, 1), (-1, 0, 1), (1, 0, -1), (-1, 0, -1), (1, 1, 1), (1, 1, -1),
         (1, -1, 1), (1, -1, -1), (-1, 1, 1), (-1, 1, -1), (-1, -1, 1), (-1, -1, -1)],
}


def _weights(q):
    """Lattice weights by speed class, as each reference file lists them."""
    e = np.array(_E[q])
    s = (e * e).sum(1)
    table = {
        13: {0: 1.0 / 2, 2: 1.0 / 24},
        15: {0: 2.0 / 9, 1: 1.0 / 9, 3: 1.0 / 72},
        19: {0: 1.0 / 3, 1: 1.0 / 18, 2: 1.0 / 36},
        27: {0: 8.0 / 27, 1: 2.0 / 27, 2: 1.0 / 54, 3: 1.0 / 216},
    }[q]
    return np.array([table[int(k)] for k in s], dtype=np.float64)


def velocity_set(q):
    """(e[Q,3] int, w[Q] float64, rev[Q] int) for D3Q{q}.

    ``rev`` maps each direction to the one with negated velocity, as the
    reference builds ``vertex_reverse`` (e.g. flow/d3/d3q19.py:57-61)."""
    if q not in _E:
        raise ValueError("Unknown parameter type: D3Q{}".format(q))
    e = np.array(_E[q], dtype=np.int64)
    lookup = {tuple(v): i for i, v in enumerate(_E[q])}
    rev = np.array([lookup[tuple(-v)] for v in e], dtype=np.int64)
    return e, _weights(q), rev


# BoundaryCondition codes (config/base.py:17-23).
PERIODICAL = 11000
WALL = 1200
WALL_WITH_SPEED = 1201
NON_EQUILIBRIUM = 1400
FACES = ("input", "output", "back", "forward", "bottom", "top")
# face -> (axis, plane selector 0 = first / -1 = last, sign of e on that axis
# for the overridden directions).  flow/d3/base.py:198-323.
FACE_AXIS = {"input": (0, 0, 1), "output": (0, -1, -1), "back": (1, 0, 1),
             "forward": (1, -1, -1), "bottom": (2, 0, 1), "top": (2, -1, -1)}


def cs2_of(dtype):
    """cs = float32(sqrt(1/3)); cs**2 taken in the storage dtype (flow/base.py:37-39)."""
    cs = dtype(math.sqrt(1.0 / 3))
    return dtype(cs * cs)


def duct_profile(a, b, n_max=100):
    """Normalised duct-flow profile: the reference's ``cul_u`` evaluated on the
    ``init_u`` grid (flow/d3/base.py:10-37).  float64, shape [a, b]; each value
    rounded to 6 decimals as ``cul_u`` does."""
    y = np.linspace(-(a - 1) / 2, (a - 1) / 2, a)
    z = np.linspace(-(b - 1) / 2, (b - 1) / 2, b)
    ha, hb = a / 2.0, b / 2.0
    n = np.arange(n_max)
    nt = 2 * n + 1
    base = 32 * (-1.0) ** (n + 1) / (nt ** 3 * np.pi ** 3)
    out = np.empty((a, b), dtype=np.float64)
    for i, yy in enumerate(y):
        for j, zz in enumerate(z):
            s = np.sum(base * np.cos(nt * np.pi * yy / (2 * ha))
                       * (np.cosh(nt * np.pi * zz / (2 * ha)) / np.cosh(nt * np.pi * hb / (2 * ha))))
            out[i, j] = round(1 - (yy / ha) ** 2 + s, 6)
    return out


class OracleFlow:
    """Restatement of ``FlowD3`` (flow/d3/base.py:57-323) on numpy arrays.

    Arrays use the reference layout: f[X,Y,Z,Q], u[X,Y,Z,3], rou[X,Y,Z,1],
    FOL[X,Y,Z,3], with X,Y,Z = size+1 (flow/d3/base.py:81-82).
    """

    def __init__(self, q, size, mu, faces=None, face_uw=None, Re=10.0, dtype=np.float32, tau=None):
        self.q = q
        self.dtype = dtype
        e, w, rev = velocity_set(q)
        self.e_int = e
        self.e = e.astype(dtype)
        self.w = w.astype(dtype)
        self.rev = rev
        self.size = np.array(size, dtype=np.int64)
        self.shape = tuple(int(s) + 1 for s in size)
        self.mu = float(mu)
        self.Re = float(Re)
        faces = dict(faces or {})
        self.faces = {k: int(faces.get(k, WALL)) for k in FACES}
        for k in ("back", "forward", "bottom", "top"):
            if self.faces[k] not in (PERIODICAL, WALL, WALL_WITH_SPEED):
                raise NotImplementedError(k)
        for k in ("input", "output"):
            if self.faces[k] not in (PERIODICAL, WALL, WALL_WITH_SPEED, NON_EQUILIBRIUM):
                raise NotImplementedError(k)
        self.face_uw = {k: np.asarray((face_uw or {}).get(k, (0.0, 0.0, 0.0)), dtype=dtype)
                        for k in FACES}
        self.cs2 = cs2_of(dtype)
        # flow/d3/base.py:96; `tau` overrides it (an FP64 run with the float32
        # relaxation time of the run it is compared with)
        self.tau = dtype(3 * self.mu + 0.5) if tau is None else dtype(tau)
        self._profile = None

    # -- flow/d3/base.py:72-101 ------------------------------------------
    def init(self, f0=None):
        X, Y, Z = self.shape
        dt = self.dtype
        self.u = np.zeros((X, Y, Z, 3), dt)
        self.rou = np.ones((X, Y, Z, 1), dt)
        self.FOL = np.zeros((X, Y, Z, 3), dt)
        self.p = np.zeros((X, Y, Z, 1), dt)
        self.f = (self.rou * self.w[None, None, None, :]).astype(dt)
        self.feq = np.zeros_like(self.f)
        self.update_u_rou()
        if f0 is not None:
            # Initial-field extension: replace f after FlowD3.init, then refresh
            # the moments so the first collision sees them.
            self.f = np.array(f0, dtype=dt).copy()
            self.update_u_rou()

    # -- flow/d3/base.py:150-159 -----------------------------------------
    def cul_equ(self):
        dt = self.dtype
        tmp = (self.u @ self.e.T) / self.cs2
        nrm = np.sqrt((self.u * self.u).sum(-1, keepdims=True, dtype=dt)).astype(dt)
        u2 = nrm ** 2 / self.cs2 / dt(2)
        self.feq = ((dt(1) + tmp + tmp ** 2 / dt(2) - u2) * (self.rou * self.w)).astype(dt)
        self.f = (self.f - (self.f - self.feq) / self.tau).astype(dt)

    # -- flow/d3/base.py:161-323 -----------------------------------------
    def f_stream(self):
        fcopy = self.f.copy()
        out = self.f.copy()
        for k in range(1, self.q):
            v = fcopy[..., k]
            for a in range(3):
                s = int(self.e_int[k, a])
                if s:
                    v = np.roll(v, s, axis=a)
            out[..., k] = v
        self.f = out
        for face in FACES:              # order matters: last override wins
            self._override(face, fcopy)

    def _override(self, face, fcopy):
        axis, plane, sign = FACE_AXIS[face]
        code = self.faces[face]
        idx = [k for k in range(self.q) if self.e_int[k, axis] == sign]
        sl_t = [slice(None)] * 3
        sl_t[axis] = slice(0, 1) if plane == 0 else slice(-1, None)
        sl_t = tuple(sl_t)
        if code == PERIODICAL:
            sl_s = [slice(None)] * 3
            sl_s[axis] = slice(-1, None) if plane == 0 else slice(0, 1)
            self.f[sl_t + (idx,)] = fcopy[tuple(sl_s) + (idx,)]
        elif code == WALL:
            self.f[sl_t + (idx,)] = fcopy[sl_t + (list(self.rev[idx]),)]
        elif code == WALL_WITH_SPEED:
            dt = self.dtype
            tmp = dt(2) * (self.rou[sl_t] * self.w[idx])
            tmp = tmp * (self.e[idx] @ self.face_uw[face]) / self.cs2
            self.f[sl_t + (idx,)] = (fcopy[sl_t + (list(self.rev[idx]),)] - tmp).astype(dt)
        elif code == NON_EQUILIBRIUM and axis == 0:
            nb = slice(1, 2) if plane == 0 else slice(-2, -1)
            self.f[sl_t] = self.feq[sl_t] + (self.f[nb] - self.feq[nb])
        else:
            raise NotImplementedError(face)

    # -- flow/d3/base.py:116-148 -----------------------------------------
    def update_u_rou(self):
        dt = self.dtype
        self.rou = self.f.sum(-1, keepdims=True, dtype=dt)
        self.p = self.rou / dt(3.0)
        self.u = ((self.f @ self.e + self.FOL / dt(2.0)) / self.rou).astype(dt)
        for a in range(3):
            for pl in (0, -1):
                sl = [slice(None)] * 3
                sl[a] = pl
                self.u[tuple(sl)] = 0
        if self.faces["input"] == NON_EQUILIBRIUM:
            X, Y, Z = self.shape
            rmax = self.rou.max()
            uw = (dt(1) / rmax) * dt(self.Re * self.mu) / dt(min(Y, Z))
            if self._profile is None:
                self._profile = duct_profile(Y, Z)
            self.u[0, :, :, 0] = (float(uw) * self._profile).astype(dt)
            self.rou[0] = self.rou[1]
        if self.faces["output"] == NON_EQUILIBRIUM:
            self.rou[-1] = self.rou[-2]
            self.u[-1] = self.u[-2]

    # -- flow/d3/base.py:103-114 -----------------------------------------
    def cul_equ2(self):
        dt = self.dtype
        cs4 = dt(self.cs2 * self.cs2)
        c = dt(1) - dt(1) / (dt(2) * self.tau)
        for a in range(self.q):
            ea = self.e[a]
            t1 = (ea - self.u) / self.cs2
            t2 = ((self.u * ea) * ea) / cs4
            t3 = ((t1 + t2) * self.FOL).sum(-1, dtype=dt)
            self.f[..., a] = (self.f[..., a] + c * self.w[a] * t3).astype(dt)


# --------------------------------------------------------------------------
# Immersed boundary and rigid particles (lbm/lbm3d.py:32-167,
# particle/base/base.py:105-156, particle/coord.py:73-108)
# --------------------------------------------------------------------------
class OracleParticle:
    """Rigid particle state as the reference keeps it (particle/base/base.py:47-118)."""

    def __init__(self, lagrange, mass, area, inertia, rou, center, angle, dtype=np.float32):
        dt = dtype
        self.dtype = dt
        self._lagrange = np.asarray(lagrange, dt)
        n = self._lagrange.shape[0]
        self.mass = dt(mass)
        self.area = dt(area)
        self.I = np.asarray(inertia, dt)
        self.rou = float(rou)
        self.cx = np.asarray(center, dt).copy()
        self.cu = np.zeros(3, dt)
        self.cw = np.zeros(3, dt)
        self.cF = np.zeros(3, dt)
        self.cT = np.zeros(3, dt)
        self.angle = np.asarray(angle, dt).copy()
        self.lx = np.zeros((n, 3), dt)          # markers at the origin until the first update
        self.lF = np.zeros((n, 3), dt)
        self.lu = np.zeros((n, 3), dt)
        self.lm = np.full((n, 1), dt(self.area / dt(n)), dt)
        self.lrou = np.zeros((n, 1), dt)

    # particle/base/base.py:120-151
    def update_from_lar(self, dt_step, gl, rouf=1.0):
        if dt_step <= 0:
            raise ValueError("Time step must be positive")
        if rouf <= 0:
            raise ValueError("Fluid density must be positive")
        d = self.dtype
        g = np.array([gl, 0, 0], d)
        tmp = (d(1 - self.rou / rouf) * self.mass) * g
        self.cF = ((-self.lF * self.lm).sum(0, dtype=d) + tmp).astype(d)
        self.cu = (self.cu + self.cF / self.mass * d(dt_step)).astype(d)
        self.cx = (self.cx + self.cu * d(dt_step)).astype(d)
        self.cT = (-(np.cross(self.lx - self.cx, self.lF) * self.lm).sum(0, dtype=d)).astype(d)
        self.cw = (self.cw + d(0.1) * self.cT * d(dt_step) / self.I).astype(d)

    # particle/base/base.py:153-156 with particle/coord.py:87-108
    def update(self):
        self.angle = (self.angle + self.cw).astype(self.dtype)
        rot = rotvec_to_matrix(self.angle.astype(np.float64))
        pts = self._lagrange.astype(np.float64) @ rot.T
        self.lx = (pts.astype(self.dtype) + self.cx).astype(self.dtype)


def rotvec_to_matrix(v):
    """Rotation matrix of a rotation vector, via the unit quaternion
    (the map scipy's ``Rotation.from_rotvec(...).apply`` evaluates)."""
    v = np.asarray(v, np.float64)
    th = float(np.sqrt(v @ v))
    if th <= 1e-3:
        th2 = th * th
        s = 0.5 - th2 / 48 + th2 * th2 / 3840
    else:
        s = math.sin(th / 2) / th
    x, y, z = s * v
    w = math.cos(th / 2)
    n = math.sqrt(x * x + y * y + z * z + w * w)
    x, y, z, w = x / n, y / n, z / n, w / n
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def region_bounds(lx, size):
    """lbm/lbm3d.py:32-44: box [floor(x)-1, floor(x)+3) clamped to [0, size]."""
    d = lx.dtype.type
    rl = np.floor(lx) - d(1)
    rl = np.maximum(rl, d(0))
    rr = rl + d(3) + d(1)
    rr = np.minimum(rr, np.asarray(size, lx.dtype))
    return rl.astype(np.int32), rr.astype(np.int32)


def stencil_weights(box_lo, box_hi, lar):
    """lbm/lbm3d.py:46-64: normalised 4-point cosine weights over the box.

    Returns w[bx,by,bz] in the dtype of ``lar``."""
    d = lar.dtype.type
    ax = [np.arange(box_lo[a], box_hi[a]) for a in range(3)]
    X, Y, Z = np.meshgrid(*ax, indexing="ij")
    r = np.stack([X.astype(lar.dtype) - lar[0], Y.astype(lar.dtype) - lar[1],
                  Z.astype(lar.dtype) - lar[2]], -1).astype(lar.dtype)
    mask = np.all(np.abs(r) <= d(2), axis=-1, keepdims=True)
    arg = np.abs(r * d(np.pi) / d(2) / d(1))
    tmp = np.where(mask, (d(1) + np.cos(arg)) / d(4) / d(1), d(0)).astype(lar.dtype)
    w = np.prod(tmp, axis=-1, dtype=lar.dtype)
    s = w.sum(dtype=lar.dtype)
    if s > 0:
        w = (w / s).astype(lar.dtype)
    return w, s


def flow_to_lagrange(flow, particles, dt_step=1.0, step=1):
    """lbm/lbm3d.py:66-100.  Returns False when the weight-sum sentinel trips."""
    ok = True
    d = flow.dtype
    for p in particles:
        rl, rr = region_bounds(p.lx, flow.size)
        lu = np.zeros((p.lx.shape[0], 3), d)
        lrou = np.zeros((p.lx.shape[0], 1), d)
        for m in range(p.lx.shape[0]):
            lo, hi = rl[m], rr[m]
            w, _ = stencil_weights(lo, hi, p.lx[m])
            if abs(w.sum(dtype=d) - d(1)) > 1e-3 and step > 100:
                ok = False
            box = (slice(lo[0], hi[0]), slice(lo[1], hi[1]), slice(lo[2], hi[2]))
            lu[m, :] = (flow.u[box] * w[..., None]).sum(dtype=d)
            lrou[m, :] = (flow.rou[box] * w[..., None]).sum(dtype=d)
        p.lu = (p.cu + np.cross(p.cw[None, :], p.lx - p.cx)).astype(d)
        p.lF = (d(2) * lrou * (p.lu - lu) / d(dt_step)).astype(d)
        p.lrou = lrou
    return ok


def particle_to_wall(particles, size, dx=1.0):
    """lbm/lbm3d.py:121-167: spring force k0=300 on the six extreme markers.

    Duplicate marker indices resolve as the reference's indexed ``+=`` does on
    the CPU: each of the six entries reads the old value, the last write wins."""
    k0 = 300
    normals = np.array([[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1]])
    for p in particles:
        d = p.dtype
        bounds = np.concatenate([np.zeros(3, d), np.asarray(size, d)])
        ext = np.concatenate([np.argmin(p.lx, axis=0), np.argmax(p.lx, axis=0)])
        coord = p.lx[ext, [0, 1, 2, 0, 1, 2]]
        dist = (d(k0) * (d(1) - np.abs(coord - bounds) / d(2 * dx))).astype(d)
        dist = np.maximum(dist, d(0))
        if dist.max() == 0:
            continue
        old = p.lF[ext].copy()
        new = (old + normals.astype(d) * dist[:, None]).astype(d)
        for j in range(6):
            p.lF[ext[j]] = new[j]


def lagrange_to_flow(flow, particles, mode="reference"):
    """lbm/lbm3d.py:102-119.  ``reference``: FOL reset, then each box assigned
    in (particle, marker) order -- the last writer wins.  ``accumulate``: the
    same weights summed (the physical spreading operator)."""
    d = flow.dtype
    flow.FOL[...] = 0
    for p in particles:
        rl, rr = region_bounds(p.lx, flow.size)
        for m in range(p.lx.shape[0]):
            lo, hi = rl[m], rr[m]
            w, _ = stencil_weights(lo, hi, p.lx[m])
            box = (slice(lo[0], hi[0]), slice(lo[1], hi[1]), slice(lo[2], hi[2]))
            val = (w[..., None] * p.lF[m] * p.lm[m]).astype(d)
            if mode == "reference":
                flow.FOL[box] = val
            else:
                flow.FOL[box] += val


class OracleLBM:
    """Restatement of ``LBMBase.run_step`` / ``LBMD3`` (lbm/base.py:146-179,
    lbm/lbm3d.py:23-30) over an OracleFlow and OracleParticles.

    ``body_force`` is the uniform-force extension: added to FOL after the
    spreading step of every step."""

    def __init__(self, flow, particles=(), dt_step=1.0, dx=1.0, gl=0.0,
                 body_force=None, ibm_mode="reference"):
        self.flow = flow
        self.particles = list(particles)
        self.dt = dt_step
        self.dx = dx
        self.gl = gl
        self.body_force = None if body_force is None else np.asarray(body_force, flow.dtype)
        self.ibm_mode = ibm_mode
        self.step = 1
        self.run_status = True

    def init(self, f0=None):
        self.flow.init(f0)
        self.flow.cul_equ()

    def run_step(self):
        fl = self.flow
        fl.cul_equ()
        fl.f_stream()
        fl.update_u_rou()
        ok = flow_to_lagrange(fl, self.particles, self.dt, self.step)
        if not ok:
            self.run_status = False
        particle_to_wall(self.particles, fl.size, self.dx)
        for p in self.particles:
            p.update_from_lar(dt_step=self.dt, gl=self.gl)
        lagrange_to_flow(fl, self.particles, self.ibm_mode)
        if self.body_force is not None:
            fl.FOL = (fl.FOL + self.body_force).astype(fl.dtype)
        fl.cul_equ2()
        fl.update_u_rou()
        for p in self.particles:
            p.update()

    def run(self, n):
        for _ in range(n):
            self.run_step()
            if not self.run_status:
                break
            self.step += 1


# --------------------------------------------------------------------------
# Marker generation (particle/base/ellipsoid.py:10-95)
# --------------------------------------------------------------------------
def surface_markers(ra, rb, rc, dx=1.0):
    """Restatement of ``generate_uniform_points_on_ellipsoid`` over the box
    [-r-2dx, r+2dx) per axis: every cube whose 8 corners straddle the surface
    contributes the centroid of the surface crossings on all corner pairs of
    opposite sign (needs >= 3 crossings).  The crossing on each pair is solved
    in closed form (the implicit function is quadratic along the segment)
    instead of the reference's ``fsolve``; both converge to the same root."""
    inv = np.array([1.0 / ra ** 2, 1.0 / rb ** 2, 1.0 / rc ** 2])

    def val(p):
        # term by term, as the reference's implicit function is written, so
        # that corners lying exactly on the surface classify identically
        return p[:, 0] ** 2 / ra ** 2 + p[:, 1] ** 2 / rb ** 2 + p[:, 2] ** 2 / rc ** 2 - 1

    xs = np.arange(-ra - 2 * dx, ra + 2 * dx, dx)
    ys = np.arange(-rb - 2 * dx, rb + 2 * dx, dx)
    zs = np.arange(-rc - 2 * dx, rc + 2 * dx, dx)
    pts = []
    for i in range(len(xs) - 1):
        for j in range(len(ys) - 1):
            for k in range(len(zs) - 1):
                cx = (xs[i], xs[i + 1])
                cy = (ys[j], ys[j + 1])
                cz = (zs[k], zs[k + 1])
                verts = np.array([(cx[a], cy[b], cz[c]) for a in (0, 1) for b in (0, 1) for c in (0, 1)])
                inside = val(verts) < 0
                if inside.any() and not inside.all():
                    cross = []
                    for a in range(8):
                        for b in range(a + 1, 8):
                            if inside[a] != inside[b]:
                                cross.append(_segment_root(verts[a], verts[b], inv))
                    if len(cross) >= 3:
                        pts.append(np.mean(cross, axis=0))
    return np.array(pts)


def _segment_root(p1, p2, inv):
    d = p2 - p1
    A = (d * d * inv).sum()
    B = 2 * (p1 * d * inv).sum()
    C = (p1 * p1 * inv).sum() - 1
    disc = max(B * B - 4 * A * C, 0.0)
    sq = math.sqrt(disc)
    roots = [(-B - sq) / (2 * A), (-B + sq) / (2 * A)]
    t = min(roots, key=lambda r: abs(r - 0.5))
    return p1 + t * d
