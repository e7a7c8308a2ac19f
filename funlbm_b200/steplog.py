"""Per-step log of the solver, off the step loop.

The reference logs every step (``LBMBase._log_step_info``, lbm/base.py:105-144):
min / mean / max of f, u and rho (``Flow.to_json``, flow/base.py:183-206) and
each particle's state (``Particle.to_str`` / ``to_json``,
particle/base/base.py:161-188) to its logger and to a SQLite key-value store.
Done with host reads that is a device synchronisation and nine full-field
reductions per step.  Here the flow figures come from one device reduction
(``lbm_flow_stats``), the particle figures from a few tiny device
reductions, and both reach the host by one asynchronous copy into pinned
memory; a writer thread waits for the copy's event, formats the line and
writes it (logger, and optionally a SQLite file with the reference's table
layout), so the step loop never waits for the log.
"""
from __future__ import annotations

import json
import logging
import queue
import sqlite3
import threading

import torch


def particle_log_tensor(particle):
    """The 21 values ``Particle.to_str`` prints, as one float64 device tensor:
    cu, cx, cF, lF (min, mean, max), cw, centre, rotation vector."""
    lf = particle.lF
    parts = [particle.cu, particle.cx, particle.cF,
             torch.stack([lf.min(), lf.mean(), lf.max()]) if lf.numel() else torch.zeros(
                 3, device=particle.cx.device, dtype=particle.cx.dtype),
             particle.cw, particle.coord.center, particle.coord.angle]
    return torch.cat([p.reshape(-1).double() for p in parts])


def _fmt(vals):
    return ",".join("%.6f" % v for v in vals)


def particle_line(mass, v):
    """particle/base/base.py:161-175 from the 21 logged values."""
    return ("m=%.2f" % mass + "\tcu=" + _fmt(v[0:3]) + "\tcx=" + _fmt(v[3:6]) + "\tcf=" + _fmt(v[6:9])
            + "\tlF=" + _fmt(v[9:12]) + "\tcw=" + _fmt(v[12:15]) + "\tr=center=" + _fmt(v[15:18])
            + "\tangle=" + _fmt(v[18:21]))


def particle_json(mass, v):
    """particle/base/base.py:177-188 from the 21 logged values."""
    return {"m": mass, "cu": v[0:3], "cx": v[3:6], "cf": v[6:9], "lF": v[9:12], "cw": v[12:15],
            "coord": {"center": v[15:18], "angle": v[18:21]}}


def flow_json(stats):
    """flow/base.py:183-206 from the 9 statistics (min, mean, max of f, u, rho)."""
    return {"f": stats[0:3], "u": stats[3:6], "rho": stats[6:9]}


class StepStore:
    """The reference's per-step key-value store (lbm/base.py:78-82, 108-110):
    table ``flow`` keyed by step and table ``particle`` keyed by (step,
    particle number from 1), JSON values, in a SQLite file."""

    def __init__(self, path):
        self.db = sqlite3.connect(path, check_same_thread=False)
        self.db.execute("CREATE TABLE IF NOT EXISTS flow (key TEXT PRIMARY KEY, value TEXT)")
        self.db.execute("CREATE TABLE IF NOT EXISTS particle (key1 TEXT, key2 TEXT, value TEXT,"
                        " PRIMARY KEY (key1, key2))")

    def put(self, step, flow, particles):
        self.db.execute("INSERT OR REPLACE INTO flow VALUES (?, ?)", (str(step), json.dumps(flow)))
        for i, p in enumerate(particles):
            self.db.execute("INSERT OR REPLACE INTO particle VALUES (?, ?, ?)",
                            (str(step), str(i + 1), json.dumps(p)))
        self.db.commit()

    def close(self):
        self.db.close()


class StepLogWriter:
    """Queue of logged steps drained by one writer thread."""

    def __init__(self, logger: logging.Logger, store: StepStore = None, depth: int = 64):
        self.logger = logger
        self.store = store
        self.q = queue.Queue(maxsize=depth)
        self.lines = 0
        self.error = None
        self.thread = threading.Thread(target=self._run, name="funlbm-steplog", daemon=True)
        self.thread.start()

    def submit(self, step, flow_stats, particle_values, masses):
        """flow_stats: device float64 [9]; particle_values: device float64
        [P * 21] or None; masses: host floats.  Returns at once (the queue
        holds `depth` steps; a full queue waits for the writer)."""
        dev = flow_stats if particle_values is None else torch.cat([flow_stats, particle_values])
        host = torch.empty(dev.shape, dtype=torch.float64, pin_memory=True)
        host.copy_(dev, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        self.q.put((step, host, ev, list(masses)))

    def _run(self):
        while True:
            item = self.q.get()
            try:
                if item is None:
                    return
                step, host, ev, masses = item
                ev.synchronize()
                v = host.tolist()
                flow = flow_json(v[:9])
                info = ["step=%6d" % step, "f=" + _fmt(flow["f"]), "u=" + _fmt(flow["u"]),
                        "rho=" + _fmt(flow["rho"])]
                plist = []
                for i, m in enumerate(masses):
                    pv = v[9 + 21 * i: 9 + 21 * (i + 1)]
                    info.append(particle_line(m, pv))
                    plist.append(particle_json(m, pv))
                self.logger.info("\t".join(info))
                if self.store is not None:
                    self.store.put(step, flow, plist)
                self.lines += 1
            except Exception as exc:          # reported by flush()
                self.error = exc
            finally:
                self.q.task_done()

    def flush(self):
        """Wait until every submitted step is written."""
        self.q.join()
        if self.error is not None:
            err, self.error = self.error, None
            raise RuntimeError("step log writer failed: %s" % err)

    def close(self):
        self.flush()
        self.q.put(None)
        self.thread.join()
        if self.store is not None:
            self.store.close()
