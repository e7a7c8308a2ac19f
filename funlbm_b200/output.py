"""Headless field output: the files ``LBMD3.save_bak`` (lbm/lbm3d.py:169-244)
writes, produced without the reference's funvtk / funtecplot helpers.

* ``flow_<step>.vtk`` -- legacy VTK, binary, STRUCTURED_POINTS over the
  X x Y x Z nodes (origin 0, spacing 1) with point data ``u`` (vectors),
  ``rho`` and ``p`` (the reference hands rho and p to its VTK helper as
  cell data of the same node grid; as point data they keep their node
  positions);
* ``particle_<i>_<step>.vtk`` -- legacy VTK POLYDATA of a particle's markers
  (vertices at ``lx``) with the point scalar ``u`` = the first component of
  ``lu``, as the reference records it;
* ``tecplot_flow_{u,rho,p}_<step>.dat`` -- Tecplot ASCII, ZONE I/J/K F=POINT,
  variables x, y, z and the field's components (ux, uy, uz / rho / p).

Device fields reach the host through one pinned asynchronous copy per field;
``AsyncWriter`` writes the files on a background thread so the step loop does
not wait for the disk.
"""
from __future__ import annotations

import os
import queue
import threading

import numpy as np
import torch


def _host(t):
    """Pinned host copy of a device tensor (float32 for float fields)."""
    src = t.detach()
    if src.is_floating_point() and src.dtype != torch.float32:
        src = src.float()
    out = torch.empty(src.shape, dtype=src.dtype, pin_memory=src.is_cuda)
    out.copy_(src, non_blocking=src.is_cuda)
    return out


def write_vtk_flow(path, u, rho, p, title="flow"):
    """Legacy binary VTK of node fields u [X, Y, Z, 3], rho / p [X, Y, Z(, 1)].
    VTK orders points x fastest, so the [x][y][z] arrays are transposed."""
    u = np.asarray(u, np.float32)
    X, Y, Z = u.shape[:3]
    rho = np.asarray(rho, np.float32).reshape(X, Y, Z)
    p = np.asarray(p, np.float32).reshape(X, Y, Z)
    n = X * Y * Z
    with open(path, "wb") as fh:
        fh.write(b"# vtk DataFile Version 3.0\n")
        fh.write(("%s\nBINARY\nDATASET STRUCTURED_POINTS\n" % title[:255]).encode())
        fh.write(("DIMENSIONS %d %d %d\nORIGIN 0 0 0\nSPACING 1 1 1\n" % (X, Y, Z)).encode())
        fh.write(("POINT_DATA %d\n" % n).encode())
        fh.write(b"VECTORS u float\n")
        fh.write(np.ascontiguousarray(u.transpose(2, 1, 0, 3)).astype(">f4").tobytes())
        for name, a in (("rho", rho), ("p", p)):
            fh.write(("\nSCALARS %s float 1\nLOOKUP_TABLE default\n" % name).encode())
            fh.write(np.ascontiguousarray(a.transpose(2, 1, 0)).astype(">f4").tobytes())
        fh.write(b"\n")


def write_vtk_points(path, lx, values, name="u", title="particle"):
    """Legacy binary VTK POLYDATA: one vertex per marker with a point scalar."""
    lx = np.asarray(lx, np.float32).reshape(-1, 3)
    values = np.asarray(values, np.float32).reshape(-1)
    m = lx.shape[0]
    with open(path, "wb") as fh:
        fh.write(b"# vtk DataFile Version 3.0\n")
        fh.write(("%s\nBINARY\nDATASET POLYDATA\n" % title[:255]).encode())
        fh.write(("POINTS %d float\n" % m).encode())
        fh.write(lx.astype(">f4").tobytes())
        fh.write(("\nVERTICES %d %d\n" % (m, 2 * m)).encode())
        cells = np.stack([np.ones(m, np.int32), np.arange(m, dtype=np.int32)], 1)
        fh.write(cells.astype(">i4").tobytes())
        fh.write(("\nPOINT_DATA %d\nSCALARS %s float 1\nLOOKUP_TABLE default\n" % (m, name)).encode())
        fh.write(values.astype(">f4").tobytes())
        fh.write(b"\n")


def write_tecplot_points(path, data, variables, title="flow_u"):
    """Tecplot ASCII, point format: one line per node, x y z then the
    field's components; I runs over x fastest as Tecplot orders a zone."""
    data = np.asarray(data, np.float32)
    X, Y, Z = data.shape[:3]
    vals = data.reshape(X, Y, Z, -1)
    zz, yy, xx = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    vt = vals.transpose(2, 1, 0, 3).reshape(-1, vals.shape[3])
    table = np.column_stack([xx.reshape(-1), yy.reshape(-1), zz.reshape(-1)]
                            + [vt[:, k] for k in range(vt.shape[1])])
    with open(path, "w") as fh:
        fh.write('TITLE = "%s"\n' % title)
        fh.write("VARIABLES = " + ", ".join('"%s"' % v for v in variables) + "\n")
        fh.write("ZONE I=%d, J=%d, K=%d, F=POINT\n" % (X, Y, Z))
        fmt = " ".join(["%d"] * 3 + ["%.8e"] * vt.shape[1])
        np.savetxt(fh, table, fmt=fmt)


def snapshot(lbm):
    """Pinned host copies of everything save_bak writes (started now,
    complete when the returned event is)."""
    fl = lbm.flow
    snap = {"u": _host(fl.u), "rho": _host(fl.rou), "p": _host(fl.p), "particles": []}
    for part in lbm.particle_swarm.particles:
        snap["particles"].append((_host(part.lx), _host(part.lu[:, 0])))
    ev = torch.cuda.Event() if torch.cuda.is_available() else None
    if ev is not None:
        ev.record()
    return snap, ev


def write_snapshot(snap, step, vtk_dir, tecplot_dir):
    """The files of save_bak for one step (paths as the reference names them)."""
    s = str(step).zfill(10)
    u, rho, p = snap["u"].numpy(), snap["rho"].numpy(), snap["p"].numpy()
    write_tecplot_points(os.path.join(tecplot_dir, "tecplot_flow_u_%s.dat" % s), u,
                         ["x", "y", "z", "ux", "uy", "uz"])
    write_tecplot_points(os.path.join(tecplot_dir, "tecplot_flow_rho_%s.dat" % s), rho,
                         ["x", "y", "z", "rho"])
    write_tecplot_points(os.path.join(tecplot_dir, "tecplot_flow_p_%s.dat" % s), p,
                         ["x", "y", "z", "p"])
    write_vtk_flow(os.path.join(vtk_dir, "flow_%s.vtk" % s), u, rho, p)
    for i, (lx, lu0) in enumerate(snap["particles"]):
        write_vtk_points(os.path.join(vtk_dir, "particle_%s_%s.vtk" % (str(i).zfill(3), s)),
                         lx.numpy(), lu0.numpy())


class AsyncWriter:
    """One background thread that writes queued snapshots in order."""

    def __init__(self):
        self.q = queue.Queue(maxsize=4)
        self.error = None
        self.thread = threading.Thread(target=self._run, name="funlbm-output", daemon=True)
        self.thread.start()

    def submit(self, snap, ev, step, vtk_dir, tecplot_dir):
        self.q.put((snap, ev, step, vtk_dir, tecplot_dir))

    def _run(self):
        while True:
            item = self.q.get()
            try:
                if item is None:
                    return
                snap, ev, step, vtk_dir, tecplot_dir = item
                if ev is not None:
                    ev.synchronize()
                write_snapshot(snap, step, vtk_dir, tecplot_dir)
            except Exception as exc:
                self.error = exc
            finally:
                self.q.task_done()

    def flush(self):
        self.q.join()
        if self.error is not None:
            err, self.error = self.error, None
            raise RuntimeError("field output failed: %s" % err)
