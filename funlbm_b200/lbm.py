"""Solver driver with the reference's API (funlbm ``lbm/base.py``, ``lbm/lbm3d.py``).

``Config``, ``LBMBase``, ``LBMD3`` (+ ``LBMD3Q13/15/19/27``) and
``create_lbm_config``.  ``LBMD3.run_step`` is the fused path:

* no particles -- one kernel per step (stream, moments, forcing, moments,
  collide of ``lbm/base.py:159-175`` plus the next step's ``cul_equ``);
* particles -- interpolation (fused with the moment pass it reads and the
  wall spring), spreading, the Newton-Euler update fused with the marker
  update, the fused step: four C-ABI calls per step.  The particle update
  runs before the flow step (the reference runs it after): neither reads
  the other's results, so the state is the reference's.

NON_EQUILIBRIUM faces, or ``"fused": false`` in the config, run the
reference's call sequence instead (``_compute_flow`` ->
``_handle_immersed_boundary`` -> ``_update_particles``), each method one
kernel.  Keys added to the reference's config: ``fused`` (default true),
``log_per_steps`` (cadence of ``_log_step_info``; default 1 like the
reference, which logs every step), ``graph_steps`` (``run`` replays the
fused steps between logging / checkpoint steps from captured CUDA graphs of
up to this many steps; default 32, 0 = never), ``ibm.mode`` (``reference`` = the
reference's last-writer-wins spreading, ``accumulate`` = summed spreading),
``ibm.spread`` (``claims`` = global per-node claims, the default; ``tiles`` =
8^3 tiles resolved in shared memory; the same field),
``flow.precision.storage``, ``flow.body_force``, ``flow.init_field``,
``log.db`` (a SQLite file for the per-step records the reference keeps in
its key-value store; default none).  Logging at the cadence runs off the
step loop (funlbm_b200.steplog); ``save_bak`` writes the reference's VTK /
Tecplot files headlessly (funlbm_b200.output).
"""
from __future__ import annotations

import ctypes
import logging
import os
from typing import List

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .config import BaseConfig, FileConfig, deep_get
from .flow import FlowConfig, FlowD3, create_flow
from .lattice import ctypes_ref, make_force
from .particle import ParticleConfig, ParticleSwarm, create_particle_swarm
from .steplog import StepLogWriter, StepStore, particle_log_tensor

logger = logging.getLogger("funlbm_b200")


class Config(BaseConfig):
    """lbm/base.py:17-40 plus the keys listed in the module docstring."""

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self.dt: float = 1.0
        self.dx: float = 1.0
        self.checkpoint = None
        self.max_step = 10000
        self.device: str = "auto"
        self.file_config = FileConfig()
        self.flow_config = FlowConfig()
        self.particles: List[ParticleConfig] = []
        self.fused = True
        self.log_per_steps = 1
        self.ibm_mode = "reference"
        self.graph_steps = 32
        self.log_db = None
        self.ibm_spread = "claims"

    def _from_json(self, config_json: dict, *args, **kwargs) -> "Config":
        self.dt = deep_get(config_json, "dt") or self.dt
        self.dx = deep_get(config_json, "dx") or self.dx
        self.device = deep_get(config_json, "device") or self.device
        self.max_step = deep_get(config_json, "max_step") or self.max_step
        self.checkpoint = deep_get(config_json, "checkpoint") or self.checkpoint
        self.file_config = FileConfig().from_json(deep_get(config_json, "file") or {})
        self.flow_config = FlowConfig().from_json(deep_get(config_json, "flow") or {})
        prec = deep_get(config_json, "precision.storage")
        if prec:
            self.flow_config.storage = prec
        for config in deep_get(config_json, "particles") or []:
            self.particles.append(ParticleConfig().from_json(config_json=config))
        fused = deep_get(config_json, "fused")
        self.fused = True if fused is None else bool(fused)
        self.log_per_steps = int(deep_get(config_json, "log_per_steps") or self.log_per_steps)
        gs = deep_get(config_json, "graph_steps")
        self.graph_steps = self.graph_steps if gs is None else int(gs)
        self.log_db = deep_get(config_json, "log.db") or self.log_db
        self.ibm_spread = deep_get(config_json, "ibm.spread") or self.ibm_spread
        if self.ibm_spread not in ("claims", "tiles"):
            raise ValueError("ibm.spread must be 'claims' or 'tiles'")
        self.ibm_mode = deep_get(config_json, "ibm.mode") or self.ibm_mode
        if self.ibm_mode not in ("reference", "accumulate"):
            raise ValueError("ibm.mode must be 'reference' or 'accumulate'")
        return self


def create_lbm_config(path="./config.json") -> Config:
    return Config().from_file(path)


def _device_of(config):
    dev = config.device
    if dev in (None, "auto", "cpu", "mps"):
        # the build is CUDA-only: "auto" (and the reference's cpu / mps
        # choices) resolve to the current CUDA device
        if not torch.cuda.is_available():
            raise RuntimeError("funlbm_b200 needs a CUDA device (there is no CPU path)")
        return torch.device("cuda")
    return torch.device(dev)


class LBMBase:
    """lbm/base.py:47-227"""

    def __init__(self, config: Config = None, flow: FlowD3 = None,
                 particle_swarm: ParticleSwarm = None, *args, **kwargs):
        self.config: Config = config or create_lbm_config()
        self.device = _device_of(self.config)
        self.step = 1
        self.flow = flow or create_flow(flow_config=self.config.flow_config, device=self.device)
        pdt = torch.float64 if self.config.flow_config.storage == "fp64" else torch.float32
        self.particle_swarm = particle_swarm or create_particle_swarm(
            self.config.particles, device=self.device, dtype=pdt)
        self.run_status = True
        self.status_word = 0
        self._g_old = (0.0, 0.0, 0.0)
        self._fol = None
        logger.info("Running on device: %s", self.device)

    # -- main loop (lbm/base.py:86-103) ------------------------------------------
    def run(self, max_steps: int = 1000000, *args, **kwargs) -> None:
        self.init()
        total_steps = min(max_steps, self.config.max_step)
        self._run_loop(total_steps)
        self.flush_log()

    def run_steps(self, count: int) -> None:
        """Advance ``count`` steps from ``self.step`` the way ``run`` does
        (logging, checkpoints and status at their cadence, graph replays in
        between) and leave ``self.step`` at the next step."""
        if count <= 0:
            return
        last = self.step + count - 1
        self._run_loop(last)
        if self.run_status:
            self.step = last + 1

    def _run_loop(self, last):
        while True:
            quiet = self._quiet_steps(last)
            if quiet >= 2:
                self._advance_graphed(quiet)
            self.run_step(step=self.step)
            self._log_step_info(self.step)
            if self.run_status is False:
                break
            if self.step >= last:
                break
            self.step += 1

    def _quiet_steps(self, last):
        """How many steps from self.step on are plain fused steps: not the
        first (it enters the fused form, or the state a checkpoint restored
        in it), no logging, no checkpoint, not the last one."""
        gs = int(self.config.graph_steps or 0)
        if (gs < 2 or self.step <= 1 or not self._use_fused() or self.flow._mode != "fused"
                or getattr(self.flow, "_loaded_fused", False)):
            return 0
        s = self.step
        L = max(1, int(self.config.log_per_steps))
        P = max(1, int(self.config.file_config.per_steps))
        nxt = min(last, -(-s // L) * L, -(-s // P) * P)
        return max(0, nxt - s)

    def _advance_graphed(self, count):
        """Run `count` plain fused steps from captured graphs of up to
        ``graph_steps`` steps (separate graphs before and after step 100, where
        the interpolation's weight-sum check switches on: lbm/lbm3d.py:84),
        eager steps for what is left over."""
        end = self.step + count
        while self.step < end:
            rem = end - self.step
            span = rem if self.step > 100 else min(rem, 101 - self.step)
            n = min(int(self.config.graph_steps), span)
            n -= n % 2
            if n >= 2:
                g = self._graph(n)
                reps = span // n
                for _ in range(reps):
                    g.replay()
                self.step += n * reps
            else:
                self._fused_step()
                self.step += 1

    def _graph(self, n):
        """Captured n-step graph (n even) for the current buffer parity and
        interpolation phase; the Python bookkeeping returns to the same
        buffers after an even number of steps, so it replays any number of
        times.  Captured on a side stream; nothing runs during capture."""
        lat = self.flow.lattice
        # the uniform forces are baked into the captured launches, so they
        # are part of the key (a changed body force captures a new graph)
        key = (n, self.step > 100, lat.cur, getattr(self, "_fi", 0), self.body_force,
               tuple(self._g_old))
        cache = self.__dict__.setdefault("_graphs", {})
        g = cache.get(key)
        if g is None:
            cap = self.__dict__.get("_graph_stream")
            if cap is None:
                cap = self._graph_stream = torch.cuda.Stream(device=self.device)
            cap.wait_stream(torch.cuda.current_stream(self.device))
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(cap):
                g.capture_begin()
                try:
                    for _ in range(n):
                        self._fused_step()
                finally:
                    g.capture_end()
            cache[key] = g
        return g

    def _log_step_info(self, *args, **kwargs) -> None:
        """lbm/base.py:105-144 at the ``log_per_steps`` cadence; also reads the
        device status word (NaN / non-positive density, empty IBM stencil) and
        stops the run like the reference's weight-sum sentinel."""
        if self.step % max(1, self.config.log_per_steps):
            return
        self.check_status()
        if not logger.isEnabledFor(logging.INFO) and not self.config.log_db:
            return
        # the line (and the SQLite record) from device reductions, copied
        # asynchronously and written by a background thread
        parts = self.particle_swarm.particles
        pvals = torch.cat([particle_log_tensor(p) for p in parts]) if parts else None
        self._step_log().submit(self.step, self.flow.step_stats(), pvals,
                                [float(p.mass) for p in parts])

    def _step_log(self):
        w = self.__dict__.get("_log_writer")
        if w is None:
            store = StepStore(self.config.log_db) if self.config.log_db else None
            w = self._log_writer = StepLogWriter(logger, store)
        return w

    def flush_log(self):
        """Wait until every logged step has been written."""
        w = self.__dict__.get("_log_writer")
        if w is not None:
            w.flush()

    def check_status(self):
        word = self.flow.read_status()
        if self._fol is not None and self._status_ibm is not None:
            word |= int(self._status_ibm.item())
            self._status_ibm.zero_()
        self.status_word |= word
        if word & (_lib.LBM_STATUS_RHO_BAD | _lib.LBM_STATUS_U_BAD | _lib.LBM_STATUS_STENCIL_EMPTY):
            logger.error("device status 0x%x: stopping", word)
            self.run_status = False
        return word

    def run_step(self, *args, **kwargs) -> None:
        """lbm/base.py:146-157"""
        if self._use_fused():
            self._fused_step()
        else:
            self._compute_flow()
            self._handle_immersed_boundary()
            self._update_particles()
        self.save(self.step)

    def _use_fused(self):
        lat = self.flow.lattice
        return self.config.fused and lat is not None and lat.fused

    # -- reference call sequence -----------------------------------------------
    def _compute_flow(self) -> None:
        self.flow.cul_equ(step=self.step)
        self.flow.f_stream()
        self.flow.update_u_rou(step=self.step)

    def _handle_immersed_boundary(self) -> None:
        self.flow_to_lagrange()
        self.particle_to_wall()
        for particle in self.particle_swarm.particles:
            particle.update_from_lar(dt=self.config.dt, gl=self.config.flow_config.gl)
        self.lagrange_to_flow()
        self.flow.cul_equ2()
        self.flow.update_u_rou()

    def _update_particles(self) -> None:
        self.particle_swarm.update(dt=self.config.dt)

    def init(self, *args, **kwargs) -> None:
        self._init()
        if self.config.checkpoint is not None:
            self.load_checkpoint(checkpoint_path=self.config.checkpoint)

    def _init(self, *args, **kwargs):
        raise NotImplementedError()

    def flow_to_lagrange(self, *args, **kwargs):
        raise NotImplementedError()

    def lagrange_to_flow(self, *args, **kwargs):
        raise NotImplementedError()

    def particle_to_wall(self, *args, **kwargs):
        raise NotImplementedError()

    def _fused_step(self):
        raise NotImplementedError()

    # -- checkpoints (lbm/base.py:198-227) --------------------------------------
    def save(self, step=10, *args, **kwargs):
        if step % self.config.file_config.per_steps > 0:
            return
        path = os.path.join(self.config.file_config.checkpoint_path,
                            "checkpoint_%s" % str(step).zfill(10))
        try:
            import h5py  # noqa: F401
        except ImportError:
            h5py = None
        if h5py is not None:
            with h5py.File(path + ".h5", "w") as fw:
                self.dump_checkpoint(fw)
        else:
            store = _NpzGroup()
            self.dump_checkpoint(store)
            np.savez(path + ".npz", **store.flat())

    def dump_checkpoint(self, group=None, *args, **kwargs):
        group.create_dataset("step", data=[self.step])
        self.flow.dump_checkpoint(group.create_group("flow"), *args, **kwargs)
        self.particle_swarm.dump_checkpoint(group=group.create_group("particle"), *args, **kwargs)

    def load_checkpoint(self, checkpoint_path=None, group=None, *args, **kwargs):
        if group is None:
            if checkpoint_path is None or not os.path.exists(checkpoint_path):
                logger.error("load failed, checkpoint_path and group cannot be both None.")
                return
            if checkpoint_path.endswith(".npz"):
                group = _NpzGroup.load(checkpoint_path)
            else:
                import h5py

                group = h5py.File(checkpoint_path, "r")
        self.step = int(group["step"][0])
        self.flow.load_checkpoint(group.get("flow"), *args, **kwargs)
        self.particle_swarm.load_checkpoint(group=group.get("particle"), *args, **kwargs)


class _NpzGroup:
    """Minimal h5py-group stand-in backed by a dict (``.npz`` checkpoints when
    h5py is not installed; same dataset names as the reference's layout)."""

    def __init__(self, prefix="", store=None):
        self.prefix = prefix
        self.store = {} if store is None else store

    def create_group(self, name):
        return _NpzGroup(self.prefix + name + "/", self.store)

    def create_dataset(self, name, data=None, **kwargs):
        self.store[self.prefix + name] = np.asarray(data)

    def get(self, name):
        key = self.prefix + name
        if key in self.store:
            return self.store[key]
        if any(k.startswith(key + "/") for k in self.store):
            return _NpzGroup(key + "/", self.store)
        return None

    def __getitem__(self, name):
        return self.get(name)

    def flat(self):
        return dict(self.store)

    @classmethod
    def load(cls, path):
        with np.load(path) as z:
            return cls("", {k: z[k] for k in z.files})


class LBMD3(LBMBase):
    """lbm/lbm3d.py:11-244 on liblbm_b200.so."""

    def __init__(self, *args, **kwargs):
        super().__init__(*args, **kwargs)
        self._status_ibm = None

    def _init(self):
        """lbm/lbm3d.py:23-30"""
        self.flow.init()
        self.flow.cul_equ()
        self.particle_swarm.init()
        self._g_old = (0.0, 0.0, 0.0)

    @property
    def body_force(self):
        bf = self.config.flow_config.body_force
        return (0.0, 0.0, 0.0) if bf is None else tuple(float(v) for v in bf)

    def _stream(self):
        return _lib.stream_of(torch, self.device)

    # -- IBM buffers ------------------------------------------------------------
    def _ensure_ibm(self):
        if self._fol is not None:
            return
        n = self.flow.n
        dev = self.device
        rdt = self.flow.lattice.real_dtype
        self._fol = [torch.zeros(n * 3, device=dev, dtype=rdt) for _ in range(2)]
        nch = (n + 31) // 32
        self._chunks = [torch.zeros(nch, dtype=torch.uint8, device=dev) for _ in range(2)]
        if self.config.ibm_spread == "tiles":
            # scratch of the tiled spreading (tile lists, weight sums), zeroed once
            nm = int(self.particle_swarm.struct().n_markers) if self.particle_swarm.particles else 0
            nb = _lib.load().ibm_spread_tiled_scratch_bytes(ctypes_ref(self.flow.lattice.desc), nm)
            self._spread_scratch = torch.zeros(nb, dtype=torch.uint8, device=dev)
        else:
            # claim array of the global-claim spreading, -1 between calls
            self._owner = torch.full((n,), -1, dtype=torch.int32, device=dev)
        self._fi = 0          # index of the buffer the next spread writes
        self._status_ibm = torch.zeros(1, dtype=torch.int32, device=dev)
        # FOL of the state being entered (zero after init): the next step's
        # "old" force field
        fol = self.flow._FOL.reshape(-1)
        if bool(torch.any(fol != 0)):
            self._fol[1].copy_(fol)
            self._chunks[1].fill_(1)

    # -- fused step ---------------------------------------------------------------
    def _fused_step(self):
        plan = self.fused_prepare()
        self.flow.fused_step(plan["force"], plan["new_field"], plan["g_new"], keep=plan["keep"])
        self.fused_finish(plan)

    def fused_prepare(self, launch=True):
        """Everything of a fused step that precedes the step kernel: enter the
        fused representation, and with particles interpolate, apply the wall
        spring and the Newton-Euler update and spread the marker forces.
        Returns the step's force description for the step kernel (run here by
        ``_fused_step``, or packed with other lattices by a server).  With
        launch=False only the description is computed (nothing is issued)."""
        fl = self.flow
        # (a checkpoint restored in the fused form counts as entering it)
        entering = fl._mode != "fused" or getattr(fl, "_loaded_fused", False)
        fl.enter_fused()
        lat = fl.lattice
        g_new = self.body_force
        g_old = self._g_old
        parts = self.particle_swarm.particles
        if parts or self._fol is not None or (entering and bool(torch.any(fl._FOL != 0))):
            self._ensure_ibm()
        if self._fol is None:
            force = None if (g_new == (0, 0, 0) and g_old == (0, 0, 0)) else make_force(g_old, g_new)
            return {"force": force, "new_field": None, "g_new": g_new, "keep": (), "ibm": False}
        s = self._stream()
        new, old = self._fi, self._fi ^ 1
        F_new, F_old = self._fol[new], self._fol[old]
        C_new, C_old = self._chunks[new], self._chunks[old]
        force = make_force(g_old, g_new, F_old, F_new, C_old, C_new)
        plan = {"force": force, "new_field": F_new, "g_new": g_new,
                "keep": (F_old, F_new, C_old, C_new), "ibm": True}
        if not launch:
            return plan
        dt = float(self.config.dt)
        mode = 0 if self.config.ibm_mode == "reference" else 1
        # reference-mode spreading with global claims: the claims and the
        # clearing of the buffer ride in the interpolation's launch
        claimed = bool(parts) and mode == 0 and self.config.ibm_spread != "tiles"
        if parts:
            sw = self.particle_swarm
            sw.ensure_extremes()
            st = ctypes.byref(sw.struct())
            f_int = make_force(old_uniform=g_old, old_field=F_old)
            # flow_to_lagrange and particle_to_wall in one launch
            args = (ctypes_ref(lat.desc), ptr(lat.buf[lat.cur]), ctypes_ref(f_int),
                    ptr(lat.face_rho[lat.cur]), st, dt, float(self.config.dx), int(self.step),
                    ptr(self._status_ibm))
            if claimed:
                call("ibm_interpolate_wall_claim", *args, ptr(F_new), ptr(C_new),
                     ptr(self._owner), s)
            else:
                call("ibm_interpolate_wall", *args, s)
        sw_struct = self.particle_swarm.struct() if parts else _empty_particles()
        if claimed:
            call("ibm_spread_claimed", ctypes_ref(lat.desc), ctypes.byref(sw_struct), ptr(F_new),
                 ptr(C_new), ptr(self._owner), s)
        elif self.config.ibm_spread == "tiles":
            call("ibm_spread_tiled", ctypes_ref(lat.desc), ctypes.byref(sw_struct), mode,
                 ptr(F_new), ptr(C_new), ptr(self._spread_scratch), self._spread_scratch.numel(),
                 s)
        else:
            call("ibm_spread", ctypes_ref(lat.desc), ctypes.byref(sw_struct), mode, ptr(F_new),
                 ptr(C_new), ptr(self._owner), s)
        if parts:
            # update_from_lar and Particle.update (with the next step's wall
            # markers) in one launch: nothing after spreading reads the old
            # positions, and the flow step does not read particle state
            call("rigid_step", st, dt, float(self.config.flow_config.gl), 1.0, s)
            sw.ext_valid = True
        return plan

    def fused_finish(self, plan):
        """Everything of a fused step after the step kernel: the force-buffer
        swap (the particle update ran with the IBM launches)."""
        if plan["ibm"]:
            self._fi ^= 1
        self._g_old = plan["g_new"]

    # -- reference-mode IBM methods (lbm/lbm3d.py:66-167) -------------------------
    def flow_to_lagrange(self, *args, **kwargs):
        parts = self.particle_swarm.particles
        if not parts:
            return
        fl = self.flow
        fl._to_ref()
        self._ensure_status()
        call("ibm_interpolate", ctypes_ref(fl.lattice.desc_fp32), None, None, None, ptr(fl._u),
             ptr(fl._rou), ctypes.byref(self.particle_swarm.struct()), float(self.config.dt),
             int(self.step), ptr(self._status_ibm), self._stream())

    def particle_to_wall(self, *args, **kwargs):
        if not self.particle_swarm.particles:
            return
        call("rigid_wall_and_update", ctypes_ref(self.flow.lattice.desc_fp32),
             ctypes.byref(self.particle_swarm.struct()), _lib.RIGID_WALL, float(self.config.dt),
             float(self.config.dx), float(self.config.flow_config.gl), 1.0, self._stream())

    def lagrange_to_flow(self, *args, **kwargs):
        fl = self.flow
        fl._to_ref()
        fl._FOL.zero_()
        parts = self.particle_swarm.particles
        if parts:
            if not hasattr(self, "_ref_chunks"):
                nch = (fl.n + 31) // 32
                self._ref_chunks = torch.zeros(nch, dtype=torch.uint8, device=self.device)
                self._ref_owner = torch.full((fl.n,), -1, dtype=torch.int32, device=self.device)
            self._ref_chunks.zero_()
            mode = 0 if self.config.ibm_mode == "reference" else 1
            call("ibm_spread", ctypes_ref(fl.lattice.desc_fp32),
                 ctypes.byref(self.particle_swarm.struct()), mode, ptr(fl._FOL), ptr(self._ref_chunks),
                 ptr(self._ref_owner), self._stream())
        g = self.body_force
        if g != (0.0, 0.0, 0.0):
            fl._FOL += torch.tensor(g, device=self.device, dtype=torch.float32)

    # -- field output (lbm/lbm3d.py:169-244) -------------------------------------
    def save_bak(self, step=10, *args, **kwargs):
        """The reference's VTK / Tecplot output every ``file.per_steps`` steps:
        flow u, rho, p on the nodes and each particle's markers, written by a
        background thread from pinned copies (funlbm_b200.output)."""
        if step % self.config.file_config.per_steps > 0:
            return
        from .output import AsyncWriter, snapshot

        w = self.__dict__.get("_out_writer")
        if w is None:
            w = self._out_writer = AsyncWriter()
        snap, ev = snapshot(self)
        w.submit(snap, ev, step, self.config.file_config.vtk_path,
                 self.config.file_config.tecplot_path)

    def flush_output(self):
        """Wait until every queued save_bak snapshot is on disk."""
        w = self.__dict__.get("_out_writer")
        if w is not None:
            w.flush()

    def _ensure_status(self):
        if self._status_ibm is None:
            self._status_ibm = torch.zeros(1, dtype=torch.int32, device=self.device)


_EMPTY = None


def _empty_particles():
    global _EMPTY
    if _EMPTY is None:
        _EMPTY = _lib.LbmParticles()
    return _EMPTY


class LBMD3Q27(LBMD3):
    pass


class LBMD3Q19(LBMD3):
    pass


class LBMD3Q15(LBMD3):
    pass


class LBMD3Q13(LBMD3):
    pass
