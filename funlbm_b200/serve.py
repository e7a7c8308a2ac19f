"""Serving: many independent simulations advanced together on one GPU.

``LBMServer`` takes a stream of solve requests -- each one a funlbm config
(any grid size, velocity set, storage, particles, faces) plus a step count
and an arrival time -- and runs them with continuous batching:

* **admission** -- a request is admitted as soon as it has arrived, a slot is
  free and its estimated device memory (its population buffers, moment and
  force fields and IBM buffers, plus room for the copy made while it is
  built) fits in the HBM budget; finished requests free their slot and
  memory at once;
* **resident state** -- each admitted request keeps its populations,
  particle state and IBM buffers on the device until it finishes;
* **overlapped execution (mode "streams", the default)** -- every request
  runs on the least-loaded stream of a pool, from its own captured CUDA
  graphs of up to 32 steps, enqueued in chunks a bounded distance ahead of
  the device, so the requests' kernels overlap on the GPU while requests
  join and leave;
* **multi-lattice launches (mode "batched")** -- all active lattices of one
  (velocity set, storage, nodes per thread) advance in one multi-lattice
  launch per step (``lbm_flow_step_batch``), the particle kernels of each
  lattice issued around it, two steps of the whole active set captured as
  one graph and recaptured when the set changes.

Each request's result (final rho, u and particle state) is the same as when
it runs alone through ``LBMD3.run_step``: the batched kernel runs the same
per-node code, and every launch shape gives the same bits.
"""
from __future__ import annotations

import ctypes
import itertools
import time
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional

import torch

from . import _lib
from ._lib import call, ptr
from .lattice import REAL_DTYPE, Lattice, ctypes_ref

_ids = itertools.count()


@dataclass
class Request:
    """One solve: a funlbm config dict, a step count and an arrival time (s)."""

    config: Dict[str, Any]
    steps: int
    arrival: float = 0.0
    rid: int = field(default_factory=lambda: next(_ids))
    admitted_at: Optional[float] = None
    finished_at: Optional[float] = None
    result: Optional[Dict[str, Any]] = None
    nodes: int = 0

    @property
    def latency(self):
        return None if self.finished_at is None else self.finished_at - self.arrival


def _shape_of(cfg):
    size = (cfg.get("flow") or {}).get("size") or [100, 100, 100]
    return tuple(int(s) + 1 for s in size)


def _q_storage(cfg):
    flow = cfg.get("flow") or {}
    q = int(str(flow.get("param_type") or "D3Q19")[3:])
    storage = ((flow.get("precision") or {}).get("storage")) or flow.get("storage") or "fp32"
    return q, storage


def estimate_bytes(cfg):
    """Device memory one request holds while it steps: the two population
    buffers (rows pitched), the moments / force fields kept for observation
    and, with particles, the IBM buffers.  The reference-form populations
    exist only while a request enters the fused form and while its result is
    read (transient_bytes)."""
    q, storage = _q_storage(cfg)
    X, Y, Z = _shape_of(cfg)
    n = X * Y * Z
    pops = Lattice.bytes_needed(q, (X, Y, Z), storage)
    fields = (3 + 1 + 1 + 3) * REAL_DTYPE[storage].itemsize * n     # u, rho, p, FOL
    ibm = (2 * 12 + 4) * n + 2 * (n // 32 + 1) if cfg.get("particles") else 0
    return int(pops + fields + ibm + (8 << 20))


def transient_bytes(cfg):
    """Extra device memory while a request enters the fused form or its
    result is read: the reference-form populations and one copy of them."""
    q, storage = _q_storage(cfg)
    X, Y, Z = _shape_of(cfg)
    return int(2 * q * X * Y * Z * REAL_DTYPE[storage].itemsize)


class _Slot:
    def __init__(self, req, lbm, nbytes):
        self.req = req
        self.lbm = lbm
        self.nbytes = nbytes
        self.remaining = req.steps
        self.started = False
        self.stream = None
        self.graphs = {}
        self.inflight = []


class LBMServer:
    """Continuous-batching server of LBM solves on one GPU.

    mode="streams" (default): every admitted request gets the least-loaded
    stream of a pool and its own CUDA graphs of up to `graph_steps` steps.
    Its run is enqueued in chunks of `chunk_steps` steps, at most two chunks
    ahead of the device, so the requests' work overlaps on the GPU while no
    stream holds a long backlog.  Everything that synchronises with the host
    (building the request, its first step, graph capture, reading results)
    runs on a separate, lightly loaded init stream, and completion is polled
    with events, so admitting or finishing a request never waits for the
    others' work.  Run the process with CUDA_DEVICE_MAX_CONNECTIONS=32 (set
    before CUDA starts) so that the pool's streams do not share hardware
    queues.

    mode="batched": all active lattices of one (velocity set, storage, nodes
    per thread) advance together in one multi-lattice step launch per step;
    two steps of the whole active set are captured as one graph, recaptured
    whenever the active set changes.
    """

    def __init__(self, budget_bytes=160e9, max_slots=256, device="cuda", use_graphs=True,
                 chunk=32, mode="streams", streams=31, graph_steps=32, chunk_steps=256,
                 reserve=True, tune=True):
        if mode not in ("streams", "batched"):
            raise ValueError("mode must be 'streams' or 'batched'")
        self.mode = mode
        self.tune = bool(tune)
        self.graph_steps = max(2, int(graph_steps) - int(graph_steps) % 2)
        self.chunk_steps = max(self.graph_steps, int(chunk_steps))
        self._streams = [torch.cuda.Stream(device=device) for _ in range(max(1, int(streams)))]
        self._init_stream = torch.cuda.Stream(device=device)
        self._next_stream = 0
        self.budget = int(budget_bytes)
        self.max_slots = int(max_slots)
        self.device = torch.device(device)
        self.use_graphs = use_graphs
        self.chunk = max(2, int(chunk))
        self.queue: List[Request] = []
        self.active: List[_Slot] = []
        self.done: List[Request] = []
        self.used = 0
        self._graph = None
        self._graph_key = None
        self._graph_keep = None
        self.stats = {"graph_captures": 0, "graph_replays": 0, "eager_steps": 0,
                      "batched_launches": 0, "max_active": 0, "max_used_bytes": 0,
                      "t_admit": 0.0, "t_capture": 0.0, "t_steps": 0.0, "t_retire": 0.0}
        if reserve:
            self._reserve_memory()

    def _reserve_memory(self):
        """Have the caching allocator take the budget from the device once, up
        front: later allocations are carved out of that cached segment instead
        of calling cudaMalloc, which stalls the host while the GPU is busy."""
        free, _ = torch.cuda.mem_get_info(self.device)
        nbytes = min(self.budget, free - (2 << 30))
        if nbytes > 0:
            block = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            del block

    # -- queue ---------------------------------------------------------------
    def submit(self, req: Request):
        if estimate_bytes(req.config) + transient_bytes(req.config) > self.budget:
            raise ValueError("request %d needs more device memory than the whole budget" % req.rid)
        self.queue.append(req)
        self.queue.sort(key=lambda r: r.arrival)

    def _admit(self, now):
        admitted = False
        i = 0
        while i < len(self.queue) and len(self.active) < self.max_slots:
            req = self.queue[i]
            if req.arrival > now:
                break
            nbytes = estimate_bytes(req.config)
            # room for the request and for its transient while it is built
            if self.used + nbytes + transient_bytes(req.config) > self.budget:
                i += 1                      # first fit: a smaller request may go ahead
                continue
            self.queue.pop(i)
            cfg = dict(req.config)
            cfg.setdefault("log_per_steps", 10 ** 9)
            cfg.setdefault("file", {"per_steps": 10 ** 9})
            cfg["device"] = str(self.device)
            try:
                slot = self._start(req, cfg, nbytes)
            except (ValueError, NotImplementedError, TypeError, KeyError) as e:
                # the solver refused this config (the reference's error types):
                # report it on the request and keep serving the others
                req.result = {"error": "%s: %s" % (type(e).__name__, e)}
                req.admitted_at = req.finished_at = now if now != float("inf") else 0.0
                self.done.append(req)
                self.stats["rejected"] = self.stats.get("rejected", 0) + 1
                continue
            req.admitted_at = now
            req.nodes = slot.lbm.flow.n
            self.active.append(slot)
            self.used += nbytes
            admitted = True
        self.stats["max_active"] = max(self.stats["max_active"], len(self.active))
        self.stats["max_used_bytes"] = max(self.stats["max_used_bytes"], self.used)
        return admitted

    def _start(self, req, cfg, nbytes):
        """Build one admitted request on the device (and, in streams mode, run
        its first step and enqueue its first chunks)."""
        from .lbm import LBMD3, Config

        if self.mode != "streams":
            lbm = LBMD3(config=Config().from_json(cfg))
            lbm.init()
            return _Slot(req, lbm, nbytes)
        init = self._init_stream
        with torch.cuda.stream(init):
            lbm = LBMD3(config=Config().from_json(cfg))
            lbm.init()
            slot = _Slot(req, lbm, nbytes)
            # the first step enters the fused representation (allocates)
            lbm.run_step(step=lbm.step)
            lbm.step += 1
            slot.remaining -= 1
            self.stats["eager_steps"] += 1
            self._tune(lbm)
            ready = torch.cuda.Event()
            ready.record(init)
        slot.stream = self._pick_stream()
        slot.stream.wait_event(ready)
        self._top_up(slot)
        return slot

    def prepare(self, requests):
        """Tune the launch-shape classes these requests will need, ahead of
        serving them (a running server keeps the choices cached, so only the
        first requests of a new class would otherwise pay for the tuning)."""
        if not self.tune:
            return
        from .tune import tune_class_of

        with torch.cuda.stream(self._init_stream):
            for r in requests:
                flow = r.config.get("flow") or {}
                q = int(str(flow.get("param_type") or "D3Q19")[3:])
                storage = ((flow.get("precision") or {}).get("storage")) or "fp32"
                nz = _shape_of(r.config)[2]
                forced = bool(r.config.get("particles")) or any(
                    float(v) != 0.0 for v in (flow.get("body_force") or ()))
                tune_class_of(q, storage, nz, forced, device=self.device)
        torch.cuda.synchronize(self.device)

    def _tune(self, lbm):
        """Launch shape of this request's step kernel from the autotuner (per
        class of lattice, cached), before any graph captures it."""
        if not self.tune:
            return
        from .tune import tune_class

        lat = lbm.flow.lattice
        if lat is not None and lat.fused:
            forced = bool(lbm.particle_swarm.particles) or lbm.body_force != (0, 0, 0)
            tune_class(lat, forced=forced)

    # -- streams mode --------------------------------------------------------------
    def _pick_stream(self):
        load = {id(st): 0 for st in self._streams}
        for slot in self.active:
            if slot.stream is not None:
                load[id(slot.stream)] += 1
        return min(self._streams, key=lambda st: load[id(st)])

    def _graph_for(self, slot, n):
        """The captured n-step graph of this lattice for its current buffer
        parity and interpolation phase (the weight-sum check switches on after
        step 100, lbm/lbm3d.py:84, and is a parameter of the captured
        launches); captured on the init stream the first time it is needed
        (no device synchronisation; nothing runs).  The bookkeeping returns to
        the same buffers after an even number of steps, so a graph can be
        replayed any number of times."""
        lbm = slot.lbm
        key = (n, lbm.step > 100, lbm.flow.lattice.cur, getattr(lbm, "_fi", 0))
        g = slot.graphs.get(key)
        if g is None:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(self._init_stream):
                g.capture_begin()
                try:
                    for _ in range(n):
                        lbm._fused_step()
                finally:
                    g.capture_end()
            slot.graphs[key] = g
            self.stats["graph_captures"] += 1
        return g

    def _top_up(self, slot):
        """Keep up to two chunks of `chunk_steps` steps of this request
        enqueued on its stream: graph replays (separate graphs for steps up to
        100 and after) and eager steps for an odd remainder."""
        lbm = slot.lbm
        while len(slot.inflight) < 2 and slot.remaining > 0:
            budget = self.chunk_steps
            with torch.cuda.stream(slot.stream):
                while budget > 0 and slot.remaining > 0:
                    rem = slot.remaining
                    if self.use_graphs and rem >= 2 and budget >= 2:
                        span = rem if lbm.step > 100 else min(rem, 101 - lbm.step)
                        n = min(self.graph_steps, span, budget)
                        n -= n % 2
                        if n >= 2:
                            g = self._graph_for(slot, n)
                            reps = max(1, min(span, budget) // n)
                            for _ in range(reps):
                                g.replay()
                            self.stats["graph_replays"] += reps
                            lbm.step += n * reps
                            slot.remaining -= n * reps
                            budget -= n * reps
                            continue
                    lbm.run_step(step=lbm.step)
                    lbm.step += 1
                    slot.remaining -= 1
                    budget -= 1
                    self.stats["eager_steps"] += 1
                ev = torch.cuda.Event()
                ev.record(slot.stream)
            slot.inflight.append(ev)

    def _pump_streams(self):
        """Drop completed chunks and top every request up; True if anything
        completed."""
        progressed = False
        for slot in self.active:
            while slot.inflight and slot.inflight[0].query():
                slot.inflight.pop(0)
                progressed = True
            if slot.remaining > 0 and len(slot.inflight) < 2:
                self._top_up(slot)
        return progressed

    def _retire_streams(self, now_fn):
        finished = [slot for slot in self.active if slot.remaining <= 0 and not slot.inflight]
        if not finished:
            return False
        init = self._init_stream
        for slot in finished:
            lbm = slot.lbm
            with torch.cuda.stream(init):
                res = {"rho": lbm.flow.rou.clone(), "u": lbm.flow.u.clone(),
                       "status": lbm.check_status(), "steps": lbm.step - 1}
                ps = lbm.particle_swarm.particles
                if ps:
                    res["cx"] = torch.stack([p.cx for p in ps]).clone()
                    res["cu"] = torch.stack([p.cu for p in ps]).clone()
                    res["cw"] = torch.stack([p.cw for p in ps]).clone()
                done = torch.cuda.Event()
                done.record(init)
            done.synchronize()
            slot.req.result = res
            slot.req.finished_at = now_fn()
            self.used -= slot.nbytes
            self.done.append(slot.req)
            slot.graphs = {}
            slot.lbm = None
        self.active = [slot for slot in self.active if slot not in finished]
        return True

    # -- one step of every active lattice --------------------------------------
    @staticmethod
    def _nodes_per_thread(lat):
        # two z-nodes per thread for float32 rows of even length; 16-bit
        # storage runs fastest with one node per thread
        return 2 if lat.storage == "fp32" and lat.pz % 2 == 0 and lat.pz >= 4 else 1

    def _pack_tables(self, plans):
        """Group the active lattices by (q, storage, nodes), pack their entries
        into pinned host buffers and copy them to the device (stream-ordered).
        Returns one launch description per group."""
        groups = {}
        for slot, plan in zip(self.active, plans):
            lat = slot.lbm.flow.lattice
            key = (lat.q, lat.storage, self._nodes_per_thread(lat))
            groups.setdefault(key, []).append((slot, plan))
        esize = _lib.load().lbm_batch_entry_bytes()
        launches = []
        for (q, storage, nodes), members in groups.items():
            host = torch.empty(len(members) * esize, dtype=torch.uint8, pin_memory=True)
            begin = torch.empty(len(members), dtype=torch.int32, pin_memory=True)
            total = 0
            force_any = False
            for j, (slot, plan) in enumerate(members):
                lat = slot.lbm.flow.lattice
                nb = ctypes.c_uint32(0)
                f = plan["force"]
                call("lbm_batch_pack", ctypes_ref(lat.desc), ptr(lat.buf[lat.cur]),
                     ptr(lat.buf[lat.cur ^ 1]), None if f is None else ctypes_ref(f),
                     ptr(lat.face_rho[lat.cur]), ptr(lat.face_rho[lat.cur ^ 1]), ptr(lat.status),
                     nodes, ctypes.c_void_p(host.data_ptr() + j * esize), ctypes.byref(nb))
                begin[j] = total
                total += nb.value
                force_any = force_any or f is not None
            dev = host.to(self.device, non_blocking=True)
            dbegin = begin.to(self.device, non_blocking=True)
            launches.append({"q": q, "storage": _lib.STORAGE[storage], "nodes": nodes,
                             "force": int(force_any), "entries": dev, "begin": dbegin,
                             "count": len(members), "blocks": total, "host": (host, begin),
                             "forces": [p["force"] for _, p in members]})
        return launches

    def _step_all(self, launches=None, plans=None):
        """Issue one fused step of every active lattice on the current stream:
        the particle kernels of each lattice, one multi-lattice step launch per
        group, the marker updates.  `launches` are prepared entry tables
        (already on the device); without them the tables are packed now."""
        main = torch.cuda.current_stream(self.device)
        s = _lib.stream_of(torch, self.device)
        ibm = [slot for slot in self.active if slot.lbm.particle_swarm.particles]
        side = {}
        pool = self._streams[1:] or self._streams   # streams[0] captures the batched graph
        for j, slot in enumerate(ibm):            # fork: one branch per particle lattice
            sj = pool[j % len(pool)]
            sj.wait_stream(main)
            side[id(slot)] = sj
        if plans is None:
            plans = []
            for slot in self.active:
                sj = side.get(id(slot))
                if sj is None:
                    plans.append(slot.lbm.fused_prepare())
                else:
                    with torch.cuda.stream(sj):
                        plans.append(slot.lbm.fused_prepare())
        for sj in set(side.values()):             # join before the step launches
            main.wait_stream(sj)
        if launches is None:
            launches = self._pack_tables(plans)
        for L in launches:
            call("lbm_flow_step_batch", L["q"], L["storage"], L["nodes"], L["force"],
                 ptr(L["entries"]), ptr(L["begin"]), L["count"], L["blocks"], s)
            self.stats["batched_launches"] += 1
        for sj in set(side.values()):
            sj.wait_stream(main)
        for slot, plan in zip(self.active, plans):
            fl = slot.lbm.flow
            fl.stepped_elsewhere(plan["force"], plan["new_field"], plan["g_new"], keep=plan["keep"])
            sj = side.get(id(slot))
            if sj is None:
                slot.lbm.fused_finish(plan)
            else:
                with torch.cuda.stream(sj):
                    slot.lbm.fused_finish(plan)
        for sj in set(side.values()):             # join the marker updates
            main.wait_stream(sj)
        return launches

    def _eager_step(self):
        self._step_all()
        for slot in self.active:
            slot.lbm.step += 1
            slot.remaining -= 1
            slot.started = True
        self.stats["eager_steps"] += 1

    def _graph_key_now(self):
        return tuple((slot.req.rid, slot.lbm.flow.lattice.cur, getattr(slot.lbm, "_fi", 0),
                      slot.lbm.step > 100) for slot in self.active)

    def _flip(self, plans):
        """Advance the buffer bookkeeping by one step without running it."""
        for slot, plan in zip(self.active, plans):
            slot.lbm.flow.lattice.cur ^= 1
            if plan["ibm"]:
                slot.lbm._fi ^= 1

    def _graph_pair(self):
        """Capture (once per active set) two steps of all active lattices and
        run them.  Returns the graph, or None when it was just captured (the
        capture run already advanced every lattice by two steps)."""
        key = self._graph_key_now()
        if self._graph is not None and key == self._graph_key:
            return self._graph
        self._graph = None
        tc = time.perf_counter()
        # entry tables of both steps, packed and uploaded before the capture
        tables = []
        for _ in range(2):
            plans = [slot.lbm.fused_prepare(launch=False) for slot in self.active]
            tables.append(self._pack_tables(plans))
            self._flip(plans)
        cap = self._streams[0]
        cap.wait_stream(torch.cuda.current_stream(self.device))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(cap):
            g.capture_begin()
            try:
                for t in tables:
                    self._step_all(launches=t)
            finally:
                g.capture_end()
        torch.cuda.current_stream(self.device).wait_stream(cap)
        g.replay()
        self._graph = g
        self._graph_keep = tables
        self._graph_key = self._graph_key_now()
        self.stats["graph_captures"] += 1
        self.stats["t_capture"] += time.perf_counter() - tc
        for slot in self.active:
            slot.lbm.step += 2
            slot.remaining -= 2
        return None

    def _advance(self, k):
        """Advance every active lattice by k steps."""
        done = 0
        while done < k:
            first = [slot for slot in self.active if not slot.started]
            if first or not self.use_graphs or k - done < 2:
                self._eager_step()
                done += 1
                continue
            g = self._graph_pair()
            if g is None:               # just captured: that ran two steps
                done += 2
                continue
            g.replay()
            self.stats["graph_replays"] += 1
            for slot in self.active:
                slot.lbm.step += 2
                slot.remaining -= 2
            done += 2

    def _retire(self, now_fn):
        keep = []
        finished = []
        for slot in self.active:
            if slot.remaining <= 0:
                finished.append(slot)
            else:
                keep.append(slot)
        if not finished:
            return False
        for slot in finished:
            lbm = slot.lbm
            res = {"rho": lbm.flow.rou.clone(), "u": lbm.flow.u.clone(),
                   "status": lbm.check_status(), "steps": lbm.step - 1}
            ps = lbm.particle_swarm.particles
            if ps:
                res["cx"] = torch.stack([p.cx for p in ps]).clone()
                res["cu"] = torch.stack([p.cu for p in ps]).clone()
                res["cw"] = torch.stack([p.cw for p in ps]).clone()
            slot.req.result = res
        torch.cuda.synchronize(self.device)
        t = now_fn()
        for slot in finished:
            slot.req.finished_at = t
            self.used -= slot.nbytes
            self.done.append(slot.req)
            slot.lbm = None
        self.active = keep
        self._graph = None
        return True

    # -- main loop -------------------------------------------------------------
    def run(self, requests=(), realtime=True):
        """Serve `requests` (plus anything submitted before) to completion.
        With realtime=True arrival times are honoured against the wall clock;
        otherwise every request counts as arrived at t = 0."""
        for r in requests:
            self.submit(r)
        t0 = time.perf_counter()

        def now():
            return time.perf_counter() - t0 if realtime else float("inf")

        if self.mode == "streams":
            while self.queue or self.active:
                ta = time.perf_counter()
                self._admit(now())
                self.stats["t_admit"] += time.perf_counter() - ta
                ts = time.perf_counter()
                progressed = self._pump_streams()
                tr = time.perf_counter()
                self.stats["t_steps"] += tr - ts
                retired = self._retire_streams(lambda: time.perf_counter() - t0)
                self.stats["t_retire"] += time.perf_counter() - tr
                if not retired and not progressed:
                    if self.queue and not self.active:
                        wait = self.queue[0].arrival - now()
                        time.sleep(min(max(wait, 0.0), 0.05))
                    else:
                        time.sleep(2e-4)
            torch.cuda.synchronize(self.device)
            return self.done
        while self.queue or self.active:
            ta = time.perf_counter()
            changed = self._admit(now())
            self.stats["t_admit"] += time.perf_counter() - ta
            if changed:
                self._graph = None
            if not self.active:
                if self.queue:
                    wait = self.queue[0].arrival - now()
                    if wait > 0:
                        time.sleep(min(wait, 0.05))
                continue
            k = min(self.chunk, min(slot.remaining for slot in self.active))
            ts = time.perf_counter()
            self._advance(k)
            tr = time.perf_counter()
            self.stats["t_steps"] += tr - ts
            self._retire(lambda: time.perf_counter() - t0)
            self.stats["t_retire"] += time.perf_counter() - tr
        return self.done


def storage_code(storage):
    return _lib.STORAGE[storage]
