"""Output and the command-line front end.

The VTK writer reproduces the content of the reference's Model::saveVTK
(src/model/Model.cpp:50-117): every node at X + dx and every element with its
VTK cell type, here as a legacy ASCII file written without VTK.  The CLI
efem_gpu mirrors `EFEM -f cfg.json` (src/main/main.cpp, Simulator.cpp:6-41).
"""
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import case_from_golden, golden_files, has_gpu, write_golden_case
from efem_b200 import api

CLI = os.path.join(os.path.dirname(api.LIB_PATH), "efem_gpu")
VTK_TYPES = {4: 10, 10: 24, 8: 12, 20: 25}


def read_vtk(path):
    lines = open(path).read().split("\n")
    assert lines[0].startswith("# vtk DataFile") and lines[2] == "ASCII"
    assert lines[3] == "DATASET UNSTRUCTURED_GRID"
    n = int(lines[4].split()[1])
    pts = np.array([[float(x) for x in ln.split()] for ln in lines[5:5 + n]])
    i = 5 + n
    nc = int(lines[i].split()[1])
    cells = [[int(x) for x in ln.split()] for ln in lines[i + 1:i + 1 + nc]]
    i += 1 + nc
    assert lines[i].split()[0] == "CELL_TYPES"
    types = [int(x) for x in lines[i + 1:i + 1 + nc]]
    return pts, cells, types


@pytest.mark.parametrize("path", golden_files()[::9], ids=lambda p: p.split("/")[-1][5:-4])
def test_vtk_undeformed_and_deformed(path, tmp_path):
    cfg, d = write_golden_case(path, tmp_path)
    case = case_from_golden(path)
    m = api.Model.from_json(cfg)
    out = tmp_path / "u.vtk"
    m.write_vtk(out)
    pts, cells, types = read_vtk(out)
    assert np.array_equal(pts, case.mesh.X)
    assert [c[1:] for c in cells] == case.mesh.conn.tolist()
    assert all(c[0] == case.mesh.conn.shape[1] for c in cells)
    assert set(types) == {VTK_TYPES[case.mesh.conn.shape[1]]}
    # deformed: X + u on free nodes, fixed nodes stay
    u = d["u_solve"]
    m.write_vtk(tmp_path / "d.vtk", u)
    pd, _, _ = read_vtk(tmp_path / "d.vtk")
    expect = case.mesh.X.copy()
    expect[m.dof_map()] += u.reshape(-1, 3)
    assert np.allclose(pd, expect, rtol=0, atol=1e-15)


def test_cli_usage_and_errors(tmp_path):
    assert os.path.exists(CLI), "efem_gpu is built with the library"
    r = subprocess.run([CLI, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "-f" in r.stdout
    r = subprocess.run([CLI], capture_output=True, text=True)
    assert r.returncode == 2
    r = subprocess.run([CLI, "-f", str(tmp_path / "missing.json")], capture_output=True, text=True)
    assert r.returncode == 1 and "not found" in r.stderr


@pytest.mark.gpu
def test_cli_solves_and_writes_frames(tmp_path):
    path = golden_files("cantilever_c3d4_pressure.npz")[0]
    cfg, d = write_golden_case(path, tmp_path)
    c = json.load(open(cfg))
    c["output"]["save_frame"] = True
    c["output"]["show_log"] = True
    json.dump(c, open(cfg, "w"))
    r = subprocess.run([CLI, "-f", cfg], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    line = [ln for ln in r.stdout.splitlines() if "dx=" in ln][0]
    vals = dict(kv.split("=") for kv in line.replace("[info] ", "").split(", "))
    assert float(vals["residual"]) <= 1e-6 and int(vals["j_evalutes"]) == 1
    frames = sorted(str(p) for p in (tmp_path / "results").rglob("*.vtk"))
    assert len(frames) == 2
    deformed = [f for f in frames if f.endswith("-deformed.vtk")][0]
    undeformed = [f for f in frames if f.endswith("-undeformed.vtk")][0]
    case = case_from_golden(path)
    p0, _, _ = read_vtk(undeformed)
    assert np.array_equal(p0, case.mesh.X)
    p1, _, _ = read_vtk(deformed)
    disp = (p1 - case.mesh.X).reshape(-1)
    m = api.Model.from_json(cfg)
    ref = np.zeros_like(case.mesh.X)
    ref[m.dof_map()] = d["u_solve"].reshape(-1, 3)
    assert np.linalg.norm(disp - ref.reshape(-1)) <= 1e-5 * np.linalg.norm(ref)
