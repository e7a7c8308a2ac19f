"""Host-side writers that need no GPU: the VTK / Tecplot files of save_bak
(lbm/lbm3d.py:169-244) written from host arrays and read back, and the
per-step log formatting and SQLite store (lbm/base.py:78-82, 105-144)."""
import json
import sqlite3

import numpy as np

from funlbm_b200 import output, steplog


def test_vtk_flow_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    X, Y, Z = 4, 3, 5
    u = rng.standard_normal((X, Y, Z, 3)).astype(np.float32)
    rho = rng.standard_normal((X, Y, Z, 1)).astype(np.float32)
    p = rho / 3
    path = tmp_path / "flow.vtk"
    output.write_vtk_flow(str(path), u, rho, p)
    raw = path.read_bytes()
    assert raw.startswith(b"# vtk DataFile Version 3.0\n")
    assert b"DIMENSIONS 4 3 5\n" in raw and b"POINT_DATA 60\n" in raw
    i = raw.index(b"VECTORS u float\n") + len(b"VECTORS u float\n")
    got = np.frombuffer(raw[i:i + 60 * 12], ">f4").reshape(Z, Y, X, 3).transpose(2, 1, 0, 3)
    assert np.array_equal(got, u)
    key = b"SCALARS rho float 1\nLOOKUP_TABLE default\n"
    j = raw.index(key) + len(key)
    got = np.frombuffer(raw[j:j + 60 * 4], ">f4").reshape(Z, Y, X).transpose(2, 1, 0)
    assert np.array_equal(got, rho[..., 0])


def test_vtk_points_and_tecplot(tmp_path):
    lx = np.array([[1.5, 2.0, 3.0], [4.0, 5.5, 6.0]], np.float32)
    output.write_vtk_points(str(tmp_path / "p.vtk"), lx, [0.1, -0.2])
    raw = (tmp_path / "p.vtk").read_bytes()
    i = raw.index(b"POINTS 2 float\n") + len(b"POINTS 2 float\n")
    assert np.array_equal(np.frombuffer(raw[i:i + 24], ">f4").reshape(2, 3), lx)
    assert b"VERTICES 2 4\n" in raw
    data = np.arange(2 * 3 * 2, dtype=np.float32).reshape(2, 3, 2)
    output.write_tecplot_points(str(tmp_path / "t.dat"), data, ["x", "y", "z", "rho"])
    lines = (tmp_path / "t.dat").read_text().splitlines()
    assert lines[1] == 'VARIABLES = "x", "y", "z", "rho"'
    assert lines[2] == "ZONE I=2, J=3, K=2, F=POINT"
    rows = [ln.split() for ln in lines[3:]]
    assert len(rows) == 12
    for r in rows:                                  # x fastest, value at [x, y, z]
        x, y, z = (int(v) for v in r[:3])
        assert float(r[3]) == data[x, y, z]
    assert [int(v) for v in rows[1][:3]] == [1, 0, 0]


def test_step_log_format_and_store(tmp_path):
    stats = [0.01, 0.05, 0.2, -0.1, 0.0, 0.1, 0.99, 1.0, 1.01]
    fj = steplog.flow_json(stats)
    assert fj == {"f": stats[0:3], "u": stats[3:6], "rho": stats[6:9]}
    pv = [float(i) for i in range(21)]
    line = steplog.particle_line(12.5, pv)
    assert line.startswith("m=12.50\tcu=0.000000,1.000000,2.000000\tcx=3.000000")
    assert "\tlF=9.000000,10.000000,11.000000\tcw=" in line
    pj = steplog.particle_json(12.5, pv)
    assert pj["coord"]["angle"] == [18.0, 19.0, 20.0]
    db = str(tmp_path / "s.db")
    st = steplog.StepStore(db)
    st.put(7, fj, [pj, pj])
    st.close()
    con = sqlite3.connect(db)
    assert json.loads(con.execute("SELECT value FROM flow WHERE key='7'").fetchone()[0]) == fj
    assert con.execute("SELECT COUNT(*) FROM particle WHERE key1='7'").fetchone()[0] == 2
    con.close()
