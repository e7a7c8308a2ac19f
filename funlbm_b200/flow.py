"""Flow field objects with the reference's API, computed by liblbm_b200.so.

Mirrors funlbm's ``flow/base.py`` and ``flow/d3/*.py``: ``Param``,
``FlowConfig``, ``Flow``, ``FlowD3``, ``FlowD3Q13/15/19/27`` and
``create_flow``.  The public attributes (``f, u, rou, p, feq, FOL, tau, x``)
keep the reference's shapes: ``f`` is ``[X, Y, Z, Q]`` (a view of the
structure-of-arrays buffer), ``u``/``FOL`` ``[X, Y, Z, 3]``, ``rou``/``p``
``[X, Y, Z, 1]``, with X, Y, Z = size + 1.

Two representations of the state:

* reference mode -- the tensors above are the state and the methods
  ``cul_equ``, ``f_stream``, ``update_u_rou``, ``cul_equ2`` act on them one at
  a time (one CUDA kernel each), exactly the reference's call sequence;
* fused mode -- ``LBMD3.run_step`` advances post-collision populations with
  one kernel per step; reading an attribute recomputes the reference's state
  on the device first.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .config import BaseConfig, BoundaryCondition, BoundaryConfig, FACES, deep_get
from .lattice import Lattice, cs2_float32, ctypes_ref, make_force, tau_float32

# Velocity sets in the reference's direction order (flow/d3/d3q13.py:7-21,
# d3q15.py:7-23, d3q19.py:8-28, d3q27.py:8-36) with weights by speed class
# (d3q13.py:23-39, d3q15.py:25-43, d3q19.py:30-54, d3q27.py:38-71).
_DIRS = {
    13: "000 110 1-10 101 10-1 011 01-1 -1-10 -110 -10-1 -101 0-1-1 0-11",
    15: "000 100 -100 010 0-10 001 00-1 111 -111 1-11 -1-11 11-1 -11-1 1-1-1 -1-1-1",
    19: "000 100 -100 010 0-10 001 00-1 110 -110 1-10 -1-10 011 0-11 01-1 0-1-1 101 -101 10-1 -10-1",
    27: "000 100 -100 010 0-10 001 00-1 110 -110 1-10 -1-10 011 0-11 01-1 0-1-1 101 -101 10-1 -10-1"
        " 111 11-1 1-11 1-1-1 -111 -11-1 -1-11 -1-1-1",
}
_SPEED_W = {13: {0: 1 / 2, 2: 1 / 24}, 15: {0: 2 / 9, 1: 1 / 9, 3: 1 / 72},
            19: {0: 1 / 3, 1: 1 / 18, 2: 1 / 36}, 27: {0: 8 / 27, 1: 2 / 27, 2: 1 / 54, 3: 1 / 216}}


def _parse_dirs(s):
    out = []
    for tok in s.split():
        vals, i = [], 0
        while i < len(tok):
            if tok[i] == "-":
                vals.append(-int(tok[i + 1]))
                i += 2
            else:
                vals.append(int(tok[i]))
                i += 1
        out.append(vals)
    return out


VELOCITY_SETS = {}
for _q, _s in _DIRS.items():
    _e = _parse_dirs(_s)
    VELOCITY_SETS[_q] = (_e, [_SPEED_W[_q][sum(c * c for c in v)] for v in _e])


def _device(device):
    if device is None or device == "auto":
        if not torch.cuda.is_available():
            raise RuntimeError("funlbm_b200 needs a CUDA device (there is no CPU path)")
        return torch.device("cuda")
    dev = torch.device(device)
    if dev.type != "cuda":
        raise RuntimeError("funlbm_b200 runs on CUDA devices only, got %s" % dev)
    return dev


class Param:
    """Lattice constants (flow/base.py:15-75)."""

    def __init__(self, e, w, vertex_reverse, device="cuda", *args, **kwargs):
        self.device = _device(device)
        self.vertex_reverse = list(vertex_reverse)
        self.e = torch.tensor(e, device=self.device, dtype=torch.float32)
        self.w = torch.tensor([w], device=self.device, dtype=torch.float32)
        self.cs = torch.tensor(math.sqrt(1.0 / 3), device=self.device, dtype=torch.float32)
        self._index_cache = {}

    def eT(self):
        return self.e.t()

    def vertex_index(self, axis, value):
        key = (axis, value)
        if key not in self._index_cache:
            self._index_cache[key] = [i for i, e in enumerate(self.e.tolist()) if e[axis] == value]
        return self._index_cache[key]

    def index_reverse(self, index):
        if isinstance(index, int):
            return self.vertex_reverse[index]
        return [self.vertex_reverse[i] for i in index]

    @property
    def e_dim(self):
        return self.e.shape[0]


def make_param(q, device="cuda"):
    e, w = VELOCITY_SETS[q]
    lookup = {tuple(v): i for i, v in enumerate(e)}
    rev = [lookup[tuple(-c for c in v)] for v in e]
    return Param(e=e, w=w, vertex_reverse=rev, device=device)


class FlowConfig(BaseConfig):
    """Flow configuration (flow/base.py:78-114) plus three keys the reference
    lacks: ``precision.storage`` (fp32 | fp16s | bf16s), ``body_force``
    ([fx, fy, fz] added to FOL every step after spreading) and ``init_field``
    ({"type": "taylor_green", "u0": ...} sets f = feq(1, u0) after init)."""

    def __init__(self, *args, **kwargs):
        self.size: np.ndarray = np.zeros(3)
        self.param: dict = {}
        self.param_type: str = "D3Q19"
        self.boundary: BoundaryConfig = None
        self.gl: float = 0.0
        self.Re: float = 10
        self.mu: float = 10
        self.storage: str = "fp32"
        self.body_force = None
        self.init_field = None
        super().__init__(*args, **kwargs)

    def _from_json(self, config_json: dict, *args, **kwargs):
        self.size = np.array(deep_get(config_json, "size") or [100, 100, 100], dtype=int)
        self.param = deep_get(config_json, "param") or self.param
        self.boundary = BoundaryConfig().from_json(deep_get(config_json, "boundary") or {})
        self.param_type = deep_get(config_json, "param_type") or self.param_type
        self.Re = float(deep_get(self.param, "Re") or self.Re)
        self.mu = float(deep_get(self.param, "mu") or self.mu)
        self.gl = float(deep_get(self.param, "gl") or self.gl)
        self.storage = (deep_get(config_json, "precision.storage") or deep_get(config_json, "storage")
                        or self.storage)
        bf = deep_get(config_json, "body_force")
        self.body_force = None if bf is None else [float(v) for v in bf]
        self.init_field = deep_get(config_json, "init_field")


class Flow:
    """Flow field base (flow/base.py:117-217)."""

    def __init__(self, param: Param = None, config: FlowConfig = None, device="cuda", *args, **kwargs):
        self.device = _device(device)
        self.param = param
        self.config = config

    def init(self, *args, **kwargs):
        raise NotImplementedError("not implemented")

    def __repr__(self):
        return "%s(size=%s, Re=%s, mu=%s)" % (type(self).__name__, tuple(self.config.size),
                                              self.config.Re, self.config.mu)


class FlowD3(Flow):
    """3-D flow on liblbm_b200.so (flow/d3/base.py:57-323)."""

    def __init__(self, config: FlowConfig, param: Param = None, device="cuda", *args, **kwargs):
        super().__init__(param=param, config=config, device=device)
        self._lat = None
        self._mode = None
        self._obs_valid = False
        self._last_force = None
        self._last_fields = ()
        self._tau_t = None
        self._x = None

    # -- geometry ------------------------------------------------------------
    @property
    def shape(self):
        m, n, d = (int(s) for s in self.config.size)
        return (m + 1, n + 1, d + 1)

    @property
    def q(self):
        return self.param.e_dim

    @property
    def n(self):
        X, Y, Z = self.shape
        return X * Y * Z

    @property
    def lattice(self):
        return self._lat

    def _faces(self):
        b = self.config.boundary or BoundaryConfig()
        return b.codes(), [getattr(b, k).wall_velocity() for k in FACES]

    # -- init (flow/d3/base.py:72-101) ----------------------------------------
    def init(self, *args, **kwargs):
        X, Y, Z = self.shape
        q = self.q
        codes, uw = self._faces()
        storage = self.config.storage
        re_mu = float(self.config.Re) * float(self.config.mu)
        self._lat = Lattice(q, (X, Y, Z), codes, tau_float32(self.config.mu), storage=storage,
                            face_uw=uw, re_mu=re_mu, device=self.device, allocate=False)
        dev = self.device
        self._fp64 = storage == "fp64"
        if self._fp64:
            self._init_fp64()
            return
        self._f = self.param.w.reshape(q, 1).expand(q, self.n).contiguous()
        self._f2 = None
        self._feq = None
        self._u = torch.zeros((X, Y, Z, 3), device=dev)
        self._rou = torch.ones((X, Y, Z, 1), device=dev)
        self._p = torch.zeros((X, Y, Z, 1), device=dev)
        self._FOL = torch.zeros((X, Y, Z, 3), device=dev)
        self._scratch = torch.zeros(1, device=dev)
        self._mode = "ref"
        self._obs_valid = True
        self.update_u_rou()
        if self.config.init_field:
            self._f = self.initial_field(self.config.init_field)
            self.update_u_rou()

    def initial_field(self, spec, dtype=torch.float32):
        """f = feq(rho = 1, u0) of the ``init_field`` extension (SoA, float32
        or float64)."""
        kind = (spec.get("type") if isinstance(spec, dict) else spec) or "taylor_green"
        if kind != "taylor_green":
            raise ValueError("unknown init_field type %r" % (kind,))
        u0 = float(spec.get("u0", 0.05)) if isinstance(spec, dict) else 0.05
        u = taylor_green_velocity(self.shape, u0, self.device, dtype=dtype)
        if dtype == torch.float32:
            return equilibrium_soa(self.param, u, torch.ones(self.shape + (1,), device=self.device))
        return equilibrium_soa64(self.q, u, torch.ones(self.shape + (1,), device=self.device,
                                                       dtype=dtype))

    # -- FP64 storage ------------------------------------------------------------
    # The float64 comparison run.  The per-function kernels are float32 only,
    # so in this storage the state before the first step is kept with torch
    # float64 operations, and entering the fused form applies LBMD3._init's
    # collision and step 1's collision on the device (lbm_flow_init) in
    # float64 to the initial field.
    def _init_fp64(self):
        X, Y, Z = self.shape
        q, dev, dt = self.q, self.device, torch.float64
        w = torch.tensor(VELOCITY_SETS[q][1], dtype=dt, device=dev)
        self._f = w.reshape(q, 1).expand(q, self.n).contiguous()
        self._f2 = None
        self._feq = None
        self._u = torch.zeros((X, Y, Z, 3), device=dev, dtype=dt)
        self._rou = torch.ones((X, Y, Z, 1), device=dev, dtype=dt)
        self._p = torch.zeros((X, Y, Z, 1), device=dev, dtype=dt)
        self._FOL = torch.zeros((X, Y, Z, 3), device=dev, dtype=dt)
        self._mode = "ref"
        self._obs_valid = True
        self._collisions = 0
        self._moments64()
        if self.config.init_field:
            self._f = self.initial_field(self.config.init_field, dtype=dt)
            self._moments64()

    def _moments64(self):
        """update_u_rou (flow/d3/base.py:116-133) in float64 torch operations."""
        X, Y, Z = self.shape
        e = torch.tensor(VELOCITY_SETS[self.q][0], dtype=torch.float64, device=self.device)
        rou = self._f.sum(0).view(X, Y, Z, 1)
        # (a reshape of the transposed product is a strided view: make the
        # [x][y][z][3] layout the kernels write explicit)
        u = (e.t() @ self._f).t().contiguous().view(X, Y, Z, 3)
        u = ((u + self._FOL / 2) / rou).contiguous()
        for a in range(3):
            for pl in (0, -1):
                idx = [slice(None)] * 3
                idx[a] = pl
                u[tuple(idx)] = 0
        self._rou, self._u, self._p = rou, u, rou / 3.0

    def _fp64_only_fused(self, what):
        raise NotImplementedError("%s: FP64 storage runs the fused path only" % what)

    # -- mode switches ---------------------------------------------------------
    def _to_ref(self):
        """Make the reference tensors current (recompute them from the fused state)."""
        if self._mode == "fused":
            self._materialize()
            self._mode = "ref"

    def _materialize(self):
        if self._obs_valid:
            return
        lat = self._lat
        force, fields = self._last_force
        if self._f is None:        # released while stepping in the fused form
            self._f = torch.empty((self.q, self.n), device=self.device, dtype=lat.real_dtype)
        # the kernel writes dense [x][y][z](3) arrays through the raw pointers
        if not self._rou.is_contiguous():
            self._rou = self._rou.contiguous()
        if not self._u.is_contiguous():
            self._u = self._u.contiguous()
        lat.observe(force, f=self._f, rho=self._rou, u=self._u)
        self._p = self._rou / 3.0
        new_field, new_uniform = fields
        rdt = lat.real_dtype
        # the uniform force reaches the kernels as float32
        g = torch.tensor(new_uniform, device=self.device, dtype=torch.float32).to(rdt)
        if new_field is not None:
            self._FOL = new_field.view(self.shape + (3,)) + g
        else:
            self._FOL = g.expand(self.shape + (3,)).contiguous()
        self._obs_valid = True

    def enter_fused(self):
        """Start fused stepping from the reference state: the fused kernel
        streams from post-collision populations, so apply this step's cul_equ
        (flow/d3/base.py:150-159) and hand the result to the lattice buffers."""
        if self._mode == "fused":
            return
        lat = self._lat
        if not lat.fused:
            raise NotImplementedError("NON_EQUILIBRIUM faces run in reference mode")
        if self._fp64:
            if self._collisions != 1 or bool(torch.any(self._FOL != 0)):
                self._fp64_only_fused("entering the fused form from a stepped state")
            lat.allocate()
            lat.init(self._f)
            self._release_reference_populations()
            self._mode = "fused"
            self._obs_valid = False
            return
        lat.allocate()
        post = self._f.clone()
        call("lbm_collide", ctypes_ref(lat.desc_fp32), ptr(post), ptr(self._rou), ptr(self._u),
             None, lat.stream())
        lat.load_post_collision_fp32(post)
        del post
        if lat.needs_face_rho:
            lat.face_rho[lat.cur].copy_(face_planes(self._rou.view(self.shape)))
        self._release_reference_populations()
        self._mode = "fused"
        self._obs_valid = False

    def _release_reference_populations(self):
        """The fused form keeps the state in the lattice buffers: drop the
        reference-form populations (f, feq and the streaming copy, 4-12 bytes
        per direction and node); observing the state allocates f again."""
        self._f = None
        self._f2 = None
        self._feq = None

    def fused_step(self, force, new_field=None, new_uniform=(0.0, 0.0, 0.0), keep=()):
        """One fused step on the lattice buffers (caller prepared `force`)."""
        self._lat.step(force)
        self._loaded_fused = False
        self._last_force = (force, (new_field, tuple(new_uniform)))
        self._keep = keep
        self._obs_valid = False

    def stepped_elsewhere(self, force, new_field=None, new_uniform=(0.0, 0.0, 0.0), keep=()):
        """Record a fused step whose kernel ran in a multi-lattice launch
        (the populations moved from buf[cur] to buf[cur ^ 1])."""
        self._lat.cur ^= 1
        self._last_force = (force, (new_field, tuple(new_uniform)))
        self._keep = keep
        self._obs_valid = False

    def read_status(self):
        return self._lat.read_status() if self._lat is not None and self._lat.status is not None else 0

    # -- reference methods (one kernel each) ---------------------------------
    def cul_equ(self, step=0, *args, **kwargs):
        """flow/d3/base.py:150-159"""
        if getattr(self, "_fp64", False):
            # LBMD3._init's collision, applied on the device when the fused
            # form is entered
            if self._mode != "ref" or self._collisions:
                self._fp64_only_fused("cul_equ")
            self._collisions = 1
            return
        self._to_ref()
        if self._feq is None:
            self._feq = torch.empty_like(self._f)
        call("lbm_collide", ctypes_ref(self._lat.desc_fp32), ptr(self._f), ptr(self._rou),
             ptr(self._u), ptr(self._feq), self._lat.stream())

    def f_stream(self, *args, **kwargs):
        """flow/d3/base.py:161-323"""
        if getattr(self, "_fp64", False):
            self._fp64_only_fused("f_stream")
        self._to_ref()
        if self._f2 is None:
            self._f2 = torch.empty_like(self._f)
        feq = self._feq
        if feq is None and BoundaryCondition.NON_EQUILIBRIUM.value in self._lat.faces:
            raise RuntimeError("f_stream with NON_EQUILIBRIUM faces needs a preceding cul_equ")
        call("lbm_stream", ctypes_ref(self._lat.desc_fp32), ptr(self._f), ptr(self._f2),
             ptr(self._rou), ptr(feq), self._lat.stream())
        self._f, self._f2 = self._f2, self._f

    def update_u_rou(self, step=0, *args, **kwargs):
        """flow/d3/base.py:116-148"""
        if getattr(self, "_fp64", False):
            if self._mode != "ref" or self._collisions:
                self._fp64_only_fused("update_u_rou")
            self._moments64()
            return
        self._to_ref()
        call("lbm_moments", ctypes_ref(self._lat.desc_fp32), ptr(self._f), ptr(self._FOL),
             ptr(self._rou), ptr(self._u), ptr(self._p), ptr(self._scratch), self._lat.stream())

    def update_u_rou_boundary(self, *args, **kwargs):
        """Included in update_u_rou (the moment kernel applies the face rules)."""
        self.update_u_rou()

    def cul_equ2(self, *args, **kwargs):
        """flow/d3/base.py:103-114"""
        if getattr(self, "_fp64", False):
            self._fp64_only_fused("cul_equ2")
        self._to_ref()
        call("lbm_add_force", ctypes_ref(self._lat.desc_fp32), ptr(self._f), ptr(self._u),
             ptr(self._FOL), self._lat.stream())

    # -- attributes ------------------------------------------------------------
    def _get(self, name):
        if self._mode == "fused":
            self._materialize()
        return getattr(self, name)

    def _set(self, name, value):
        self._to_ref()
        setattr(self, name, value)

    @property
    def f(self):
        X, Y, Z = self.shape
        return self._get("_f").view(self.q, X, Y, Z).permute(1, 2, 3, 0)

    @f.setter
    def f(self, value):
        self._to_ref()
        X, Y, Z = self.shape
        dt = torch.float64 if getattr(self, "_fp64", False) else torch.float32
        v = torch.as_tensor(value, dtype=dt, device=self.device).reshape(X, Y, Z, self.q)
        self._f = v.permute(3, 0, 1, 2).contiguous().view(self.q, -1)

    @property
    def u(self):
        return self._get("_u")

    @u.setter
    def u(self, value):
        self._set("_u", torch.as_tensor(value, dtype=torch.float32, device=self.device)
                  .reshape(self.shape + (3,)).contiguous())

    @property
    def rou(self):
        return self._get("_rou")

    @rou.setter
    def rou(self, value):
        self._set("_rou", torch.as_tensor(value, dtype=torch.float32, device=self.device)
                  .reshape(self.shape + (1,)).contiguous())

    @property
    def p(self):
        return self._get("_p")

    @p.setter
    def p(self, value):
        self._set("_p", torch.as_tensor(value, dtype=torch.float32, device=self.device)
                  .reshape(self.shape + (1,)).contiguous())

    @property
    def FOL(self):
        return self._get("_FOL")

    @FOL.setter
    def FOL(self, value):
        self._set("_FOL", torch.as_tensor(value, dtype=torch.float32, device=self.device)
                  .reshape(self.shape + (3,)).contiguous())

    @property
    def feq(self):
        """Equilibrium of the last ``cul_equ`` in reference mode; in fused mode
        the equilibrium of the current moments."""
        if self._mode == "ref" and self._feq is not None:
            X, Y, Z = self.shape
            return self._feq.view(self.q, X, Y, Z).permute(1, 2, 3, 0)
        X, Y, Z = self.shape
        return equilibrium_soa(self.param, self.u, self.rou).view(self.q, X, Y, Z).permute(1, 2, 3, 0)

    @property
    def tau(self):
        if self._tau_t is None:
            self._tau_t = torch.full(self.shape + (1,), tau_float32(self.config.mu),
                                     device=self.device)
        return self._tau_t

    @property
    def x(self):
        if self._x is None:
            X, Y, Z = self.shape
            ax = [torch.arange(s, device=self.device) for s in (X, Y, Z)]
            self._x = torch.stack(torch.meshgrid(*ax, indexing="ij"), dim=-1)
        return self._x

    # -- reporting (flow/base.py:183-206) ---------------------------------------
    def step_stats(self):
        """min, mean, max of f, u and rho at the end of the last step as a
        float64 device tensor of 9 values, without a host synchronisation.
        In the fused form one reduction kernel streams the populations once
        (lbm_flow_stats); otherwise the reference tensors are reduced."""
        if self._mode == "fused" and not self._obs_valid and self._last_force is not None:
            return self._lat.stats(self._last_force[0])
        vals = []
        for t in (self.f, self.u, self.rou):
            vals += [t.min(), t.double().mean(), t.max()]
        return torch.stack([v.double() for v in vals])

    def to_json(self):
        v = self.step_stats().tolist()
        return {"f": v[0:3], "u": v[3:6], "rho": v[6:9]}

    def dump_checkpoint(self, group=None, *args, **kwargs):
        """flow/base.py:208-211: ``f``; also, not in the reference's file,
        ``FOL`` (the force the end-of-step moments include) and, while the
        state lives in the lattice buffers, the stored populations themselves
        (``populations``: dense [q][x][y][z] in the storage's type, 16-bit
        forms as their raw bits; ``storage_code``; ``face_rho``), so that a
        loaded state continues bit for bit as the saved run would have: the
        buffers hold f - w_i, which f rounded to float32 does not determine."""
        if group is None:
            return
        group.create_dataset("f", data=self.f.cpu().numpy(), compression="gzip",
                             compression_opts=9)
        group.create_dataset("FOL", data=self.FOL.cpu().numpy(), compression="gzip",
                             compression_opts=9)
        if self._mode == "fused":
            lat = self._lat
            X, Y, Z = self.shape
            pop = lat.buf[lat.cur].view(lat.q, X * Y, lat.pz)[:, :, :Z].contiguous()
            if pop.element_size() == 2:
                pop = pop.view(torch.int16)
            group.create_dataset("populations", data=pop.view(lat.q, -1).cpu().numpy(),
                                 compression="gzip", compression_opts=9)
            group.create_dataset("storage_code", data=[_lib.STORAGE[lat.storage]])
            if lat.needs_face_rho:
                group.create_dataset("face_rho", data=lat.face_rho[lat.cur].cpu().numpy())

    def load_checkpoint(self, group=None, *args, **kwargs):
        """flow/base.py:213-216 (with the reference's tensor-construction
        TypeError fixed): f, then the moments; FOL when the file has it; the
        stored populations when the file has them for this lattice's storage
        (the state then continues in the fused form exactly)."""
        if group is None:
            return
        fp64 = getattr(self, "_fp64", False)
        pop, code = group.get("populations"), group.get("storage_code")
        exact = (pop is not None and code is not None and self._lat is not None
                 and int(np.asarray(code[:]).reshape(-1)[0]) == _lib.STORAGE[self._lat.storage]
                 and tuple(np.asarray(pop[:]).shape) == (self.q, self.n))
        if fp64 and not exact:
            self._fp64_only_fused("load_checkpoint")
        dt = torch.float64 if fp64 else torch.float32
        self.f = torch.tensor(np.asarray(group.get("f")[:]), dtype=dt, device=self.device)
        fol = group.get("FOL")
        if fol is not None:
            self.FOL = torch.tensor(np.asarray(fol[:]), dtype=torch.float32, device=self.device)
        self.update_u_rou()
        if not exact:
            return
        # the populations the next step streams from, as the saved run held
        # them; f / rho / u above stay the observed state until that step
        lat = self._lat
        lat.allocate()
        X, Y, Z = self.shape
        src = torch.from_numpy(np.ascontiguousarray(np.asarray(pop[:])))
        dst = lat.buf[lat.cur].view(lat.q, X * Y, lat.pz)[:, :, :Z]
        dst.copy_(src.view(dst.dtype).view(lat.q, X * Y, Z).to(self.device))
        fr = group.get("face_rho")
        if lat.needs_face_rho and fr is not None:
            lat.face_rho[lat.cur].copy_(torch.from_numpy(np.asarray(fr[:])).to(self.device))
        self._mode = "fused"
        self._obs_valid = True
        self._loaded_fused = True       # the next step enters this state's FOL


def face_planes(rho3):
    """Densities of the six face planes, concatenated in the library's order."""
    X, Y, Z = rho3.shape
    parts = [rho3[0], rho3[-1], rho3[:, 0], rho3[:, -1], rho3[:, :, 0], rho3[:, :, -1]]
    return torch.cat([p.reshape(-1) for p in parts])


def taylor_green_velocity(shape, u0, device, dtype=torch.float32):
    """u0 (sin kx cos ky cos kz, -cos kx sin ky cos kz, 0), k = 2 pi / N per axis."""
    X, Y, Z = shape
    kx, ky, kz = (2 * math.pi / s for s in (X, Y, Z))
    x = torch.arange(X, device=device, dtype=torch.float64)[:, None, None]
    y = torch.arange(Y, device=device, dtype=torch.float64)[None, :, None]
    z = torch.arange(Z, device=device, dtype=torch.float64)[None, None, :]
    ux = u0 * torch.sin(kx * x) * torch.cos(ky * y) * torch.cos(kz * z)
    uy = -u0 * torch.cos(kx * x) * torch.sin(ky * y) * torch.cos(kz * z)
    uz = torch.zeros_like(ux * uy)
    return torch.stack(torch.broadcast_tensors(ux, uy, uz), -1).to(dtype)


def equilibrium_soa(param, u, rou):
    """feq of flow/d3/base.py:152-158 as float32 SoA [Q, n]."""
    cs2 = param.cs ** 2
    tmp = torch.matmul(u, param.eT()) / cs2
    u2 = torch.linalg.norm(u, dim=-1, keepdim=True) ** 2 / cs2 / 2
    feq = (1 + tmp + tmp ** 2 / 2 - u2) * torch.matmul(rou, param.w)
    return feq.reshape(-1, param.e_dim).t().contiguous()


def equilibrium_soa64(q, u, rou):
    """feq of flow/d3/base.py:152-158 in float64 with cs^2 = 1/3 (the FP64
    comparison run), SoA [Q, n]."""
    e = torch.tensor(VELOCITY_SETS[q][0], dtype=torch.float64, device=u.device)
    w = torch.tensor([VELOCITY_SETS[q][1]], dtype=torch.float64, device=u.device)
    cs2 = math.sqrt(1.0 / 3) ** 2
    tmp = torch.matmul(u, e.t()) / cs2
    u2 = torch.linalg.norm(u, dim=-1, keepdim=True) ** 2 / cs2 / 2
    feq = (1 + tmp + tmp ** 2 / 2 - u2) * torch.matmul(rou, w)
    return feq.reshape(-1, q).t().contiguous()


class FlowD3Q13(FlowD3):
    def __init__(self, *args, device="cuda", **kwargs):
        super().__init__(param=make_param(13, device), device=device, *args, **kwargs)


class FlowD3Q15(FlowD3):
    def __init__(self, *args, device="cuda", **kwargs):
        super().__init__(param=make_param(15, device), device=device, *args, **kwargs)


class FlowD3Q19(FlowD3):
    def __init__(self, *args, device="cuda", **kwargs):
        super().__init__(param=make_param(19, device), device=device, *args, **kwargs)


class FlowD3Q27(FlowD3):
    def __init__(self, *args, device="cuda", **kwargs):
        super().__init__(param=make_param(27, device), device=device, *args, **kwargs)


def create_flow(flow_config: FlowConfig, *args, **kwargs):
    """flow/__init__.py:16-41"""
    kinds = {"D3Q27": FlowD3Q27, "D3Q19": FlowD3Q19, "D3Q15": FlowD3Q15, "D3Q13": FlowD3Q13}
    cls = kinds.get(flow_config.param_type)
    if cls is None:
        raise ValueError("Unknown parameter type: {}".format(flow_config.param_type))
    return cls(config=flow_config, *args, **kwargs)
