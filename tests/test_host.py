"""Host-side behaviour of libefem_b200.so that needs no GPU: the exported
C ABI, the JSON / mesh readers, DOF numbering, pressure-face set-up and the
approximate-Jacobian assembly, against the reference's golden outputs."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

import oracle
from conftest import ROOT, golden_files, has_gpu, write_golden_case
from efem_b200 import api, meshgen as mg


def header_symbols():
    text = open(os.path.join(ROOT, "include", "efem_gpu.h")).read()
    return sorted(set(re.findall(r"^(?:efem_status|const char\*)\s+(efem_\w+)\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = api.lib()
    names = header_symbols()
    assert len(names) >= 14
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(api.EXPORTED) | {"efem_version"}
    assert b"sm_100a" in L.efem_version()


def test_default_options_are_the_reference_defaults():
    o = api.default_options()
    assert (o.m, o.max_linesearch, o.max_iterations, o.nl_solver) == (6, 20, 0, 0)
    assert o.residual_criterion == 1e-6 and o.dx_criterion == 1e-8


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: p.split("/")[-1][5:-4])
@pytest.mark.parametrize("integration", ["full", "reduced"])
def test_json_setup_matches_reference(path, integration, tmp_path):
    """Config + mesh + constraint readers, DOF map and L (x) I3 against the reference."""
    cfg, d = write_golden_case(path, tmp_path, integration)
    m = api.Model.from_json(cfg)
    case = oracle.read_case(cfg)
    fixed = case["fixed"].astype(bool)
    assert m.n_dof == 3 * int((~fixed).sum()) == d["u"].shape[0]
    assert np.array_equal(m.dof_map(), np.nonzero(~fixed)[0])
    rp, ci, v = m.approx_jacobian_csr()
    Vv = d["v"].reshape(-1, 3)
    Kv = np.zeros_like(Vv)
    for i in range(m.n_free):
        Kv[i] = v[rp[i]:rp[i + 1]] @ Vv[ci[rp[i]:rp[i + 1]]]
    ref = d[f"Kv_{integration}"]
    assert np.linalg.norm(Kv.ravel() - ref) <= 1e-12 * np.linalg.norm(ref)
    info = m.info()
    assert info["n_faces"] == sum(len(f) for _, f in case["pressures"])


def test_array_and_json_paths_agree(tmp_path):
    path = golden_files("case_C3D10_yeoh_dpressure.npz")[0]
    from conftest import case_from_golden
    case = case_from_golden(path)
    a = api.Model.from_case(case)
    b = api.Model.from_json(case.write(str(tmp_path)))
    assert a.info() == b.info()
    ra, rb = a.approx_jacobian_csr(), b.approx_jacobian_csr()
    for x, y in zip(ra, rb):
        assert np.array_equal(x, y)


def test_max_optim_iters_alias(tmp_path):
    case = mg.small_case("C3D4", "nh", "pressure")
    case.analysis = {"max_optim_iters": 7}
    cfg = case.write(str(tmp_path))
    j = json.load(open(cfg))
    del j["analysis"]["max_solver_iters"]
    json.dump(j, open(cfg, "w"))
    assert api.Model.from_json(cfg).options.max_iterations == 7


def test_pose_and_material_ids(tmp_path):
    """Per-element material ids and a translated / scaled body."""
    case = mg.small_case("C3D8", "nh", "force")
    case.mesh.mat = np.where(np.arange(case.mesh.conn.shape[0]) % 2 == 0, 3, 4).astype(np.int64)
    case.materials = [mg.mat_nh(C10=1e5, mid=3), mg.mat_mr(mid=4), mg.mat_yeoh(mid=3)]
    cfg = case.write(str(tmp_path))
    m = api.Model.from_json(cfg)
    assert m.info()["n_elements"] == case.mesh.conn.shape[0]
    j = json.load(open(cfg))
    j["model"][0]["pose"] = [{"t": [1.0, 2.0, 3.0]}, {"s": [2.0, 2.0, 2.0]}]
    json.dump(j, open(cfg, "w"))
    m2 = api.Model.from_json(cfg)
    # scaling lengths by 2 scales L (x) I3 (V * T^T T ~ length) by 2
    rp, ci, v = m.approx_jacobian_csr()
    rp2, ci2, v2 = m2.approx_jacobian_csr()
    # the translation to ~(2, 4, 6) costs a few digits of the element geometry
    assert np.allclose(v2, 2.0 * v, rtol=1e-8, atol=1e-8 * np.abs(v).max())


def test_undefined_material_skips_elements(tmp_path):
    case = mg.small_case("C3D4", "nh", "pressure")
    case.mesh.mat = np.full(case.mesh.conn.shape[0], 9, dtype=np.int64)
    case.mesh.mat[:5] = -1
    m = api.Model.from_json(case.write(str(tmp_path)))
    info = m.info()
    assert info["n_elements_skipped"] == case.mesh.conn.shape[0] - 5 and info["n_elements"] == 5


@pytest.mark.parametrize("bad,status", [("missing_cfg", api.ERR_CONFIG), ("bad_json", api.ERR_CONFIG),
                                        ("missing_mesh", api.ERR_MESH), ("bad_face", api.ERR_FACE),
                                        ("bad_node", api.ERR_MESH)])
def test_error_codes(bad, status, tmp_path):
    case = mg.small_case("C3D4", "nh", "pressure")
    cfg = case.write(str(tmp_path))
    if bad == "missing_cfg":
        cfg = str(tmp_path / "nope.json")
    elif bad == "bad_json":
        open(cfg, "w").write("{ \"model\": [ }")
    elif bad == "missing_mesh":
        os.remove(tmp_path / "mesh.txt")
    elif bad == "bad_face":
        open(tmp_path / "pressure0.txt", "w").write("1 2 3\n")  # three nodes of no single element face
    elif bad == "bad_node":
        open(tmp_path / "fix.txt", "w").write("100000\n")
    with pytest.raises(api.EfemError) as e:
        api.Model.from_json(cfg)
    assert e.value.status == status


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU error path")
def test_compute_without_gpu_fails_loudly():
    case = mg.small_case("C3D4", "nh", "pressure")
    m = api.Model.from_case(case)
    with pytest.raises(api.EfemError) as e:
        m.residual(np.zeros(m.n_dof))
    assert e.value.status == api.ERR_NO_DEVICE


@pytest.mark.parametrize("path", golden_files("gravity_*.npz"), ids=lambda p: p.split("/")[-1][8:-4])
@pytest.mark.parametrize("integration", ["full", "reduced"])
def test_gravity_external_load_matches_reference(path, integration, tmp_path):
    """f_ext = nodal forces + M g equals -R(0) of the reference (no pressure
    faces, so the internal force at u = 0 vanishes); under reduced integration
    the mass keeps the full rule, as in the reference).  The reference's R(0)
    carries its stress rounding at F = I (a few 1e-15 N per DOF)."""
    cfg, d = write_golden_case(path, tmp_path, integration)
    m = api.Model.from_json(cfg)
    consistent = json.loads(str(d["analysis"]))["consistent_inertia"]
    assert m.options.consistent_inertia == int(consistent)
    ref = -d["r_zero"]
    assert np.linalg.norm(m.external_load() - ref) <= 1e-11 * np.linalg.norm(ref)
    from conftest import case_from_golden
    case = case_from_golden(path)
    case.integration = integration
    a = api.Model.from_case(case)
    assert np.array_equal(a.external_load(), m.external_load())


def test_gravity_mass_switch(tmp_path):
    """Changing consistent_inertia after set-up recomputes M g."""
    lumped = golden_files("gravity_C3D10_lumped.npz")[0]
    consistent = golden_files("gravity_C3D10_consistent.npz")[0]
    cfg, dl = write_golden_case(lumped, tmp_path)
    dc = np.load(consistent)
    m = api.Model.from_json(cfg)
    first = m.external_load()
    assert np.allclose(first, -dl["r_zero"], rtol=1e-12, atol=1e-13)
    m.set_options(consistent_inertia=1)
    assert np.allclose(m.external_load(), -dc["r_zero"], rtol=1e-12, atol=1e-13)
    assert not np.allclose(m.external_load(), first, rtol=1e-6, atol=0)
    m.set_options(consistent_inertia=0)
    assert np.array_equal(m.external_load(), first)


def test_gravity_strings(tmp_path):
    case = mg.small_case("C3D8", "nh", "force")
    base = api.Model.from_case(case).external_load()
    for key, g in api.GRAVITY.items():
        case.analysis = {"gravity": key}
        m = api.Model.from_json(case.write(str(tmp_path / key.replace("-", "n"))))
        f = (m.external_load() - base).reshape(-1, 3)
        axis = int(np.nonzero(g)[0][0])
        assert np.all(np.sign(f[:, axis]) == np.sign(g[axis]))
        assert np.all(np.delete(f, axis, axis=1) == 0)
    case.analysis = {"gravity": "non"}
    m = api.Model.from_json(case.write(str(tmp_path / "non")))
    assert np.array_equal(m.external_load(), base)


def test_line_search_key(tmp_path):
    case = mg.small_case("C3D8", "nh", "force")
    case.analysis = {"line_search": "armijo"}
    assert api.Model.from_json(case.write(str(tmp_path))).options.line_search == 1
    case.analysis = {"line_search": "residual"}
    assert api.Model.from_json(case.write(str(tmp_path / "b"))).options.line_search == 0
