"""The C restatement (oracle/efem_oracle.c) against the reference's own outputs.

The golden fixtures were produced by the reference sources compiled unmodified
(tests/golden/make_golden.py); these tests pin the oracle that the GPU parity
tests then use as their checker.
"""
import json

import numpy as np
import pytest

import oracle
from conftest import golden_files, write_golden_case

CASES = golden_files()


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.split("/")[-1][5:-4])
@pytest.mark.parametrize("integration", ["full", "reduced"])
def test_residual_matches_reference(path, integration, tmp_path):
    cfg, d = write_golden_case(path, tmp_path, integration)
    o = oracle.Oracle(oracle.read_case(cfg))
    r = o.residual(d["u"])
    ref = d[f"r_{integration}"]
    assert np.linalg.norm(r - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("path", golden_files("inverted_*.npz"), ids=lambda p: p.split("/")[-1][9:-4])
def test_residual_inverted_elements_matches_reference(path, tmp_path):
    """Every element inside out (J about -1/2): the reference's laws stay
    finite there (J^{-2/3} = (J^2)^{-1/3}), and the restatement follows them."""
    d0 = np.load(path)
    for integration in (["full", "reduced"] if "r_reduced" in d0.files else ["full"]):
        cfg, d = write_golden_case(path, tmp_path, integration)
        o = oracle.Oracle(oracle.read_case(cfg))
        r = o.residual(d["u"])
        ref = d[f"r_{integration}"]
        assert np.all(np.isfinite(r))
        assert np.linalg.norm(r - ref) <= 1e-12 * np.linalg.norm(ref), integration


@pytest.mark.parametrize("path", golden_files("sample_*.npz"), ids=lambda p: p.split("/")[-1][7:-4])
def test_residual_vanishes_at_reference_sample_solutions(path, tmp_path):
    """The reference's own six sample problems (their configs and files, the
    id -1 Mooney-Rivlin material, directed and follower pressure): at the
    reference's solution converged to 1e-10 N, the restatement's residual is
    as small as the reference's own stopping test allows (1.5e-10 N)."""
    from conftest import write_sample
    cfg, d = write_sample(path, tmp_path)
    o = oracle.Oracle(oracle.read_case(cfg))
    r = o.residual(d["u_tight"])
    r0 = o.residual(np.zeros_like(d["u_tight"]))
    assert np.abs(r0).max() > 0.1
    assert np.abs(r).max() <= 1.5e-10, np.abs(r).max()


def test_beam_record_oracle_follows_reference():
    """The C3D8 beam's non-converging solve: the restatement's record of
    ||r||_2 (stored in the fixture by the generator) follows the reference's
    through the seventh line search."""
    d = np.load(golden_files("config_beam_c3d8_mr_force_record.npz")[0])
    ref, ora = d["r_norm2"], d["oracle_trace"][:, 1]
    rel = np.abs(ora[:8] - ref[:8]) / ref[:8]
    assert rel.max() <= 1e-6, rel
    assert ref[8:].min() > 1e8 and ora[8:].min() > 1e8


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.split("/")[-1][5:-4])
@pytest.mark.parametrize("integration", ["full", "reduced"])
def test_approx_jacobian_matches_reference(path, integration, tmp_path):
    cfg, d = write_golden_case(path, tmp_path, integration)
    o = oracle.Oracle(oracle.read_case(cfg))
    L = o.approx_jacobian_dense()
    v = d["v"].reshape(-1, 3)
    Kv = (L @ v).ravel()  # (L (x) I3) v
    ref = d[f"Kv_{integration}"]
    assert np.linalg.norm(Kv - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.split("/")[-1][5:-4])
def test_solve_matches_reference(path, tmp_path):
    cfg, d = write_golden_case(path, tmp_path)
    o = oracle.Oracle(oracle.read_case(cfg))
    u, info = o.solve()
    ref = d["u_solve"]
    meta = json.loads(str(d["solve_meta"]))
    assert info["r_inf"] <= 1e-6
    assert np.linalg.norm(u - ref) <= 1e-6 * np.linalg.norm(ref)
    # the restatement follows the reference's iteration path on these cases
    assert abs(info["niter"] - meta["niter"]) <= 2


def test_c3d20_reduced_solve_matches_reference(tmp_path):
    for path in golden_files("case_C3D20_*.npz"):
        cfg, d = write_golden_case(path, tmp_path / path.split("/")[-1][:-4], "reduced")
        o = oracle.Oracle(oracle.read_case(cfg))
        u, info = o.solve()
        ref = d["u_solve_reduced"]
        assert np.linalg.norm(u - ref) <= 1e-6 * np.linalg.norm(ref)


def test_cantilever_c3d4_pressure(tmp_path):
    path = golden_files("cantilever_c3d4_pressure.npz")[0]
    cfg, d = write_golden_case(path, tmp_path)
    o = oracle.Oracle(oracle.read_case(cfg))
    r0 = o.residual(np.zeros(o.n_dof))
    assert np.linalg.norm(r0 - d["r_zero"]) <= 1e-12 * np.linalg.norm(d["r_zero"])
    u, info = o.solve()
    assert np.linalg.norm(u - d["u_solve"]) <= 1e-6 * np.linalg.norm(d["u_solve"])


@pytest.mark.parametrize("mat,mtype", [("nh", 0), ("mr", 1), ("yeoh", 2)])
def test_piola_matches_reference(mat, mtype):
    d = np.load(golden_files(f"piola_{mat}.npz")[0])
    P = oracle.piola(mtype, d["C"], d["F"])
    assert np.abs(P - d["P"]).max() <= 1e-10 * np.abs(d["P"]).max()
    kappa = oracle.lib().orc_elasticity_coeff(mtype, d["C"].ctypes.data_as(oracle.ctypes.POINTER(oracle.ctypes.c_double)))
    assert kappa == pytest.approx(float(d["kappa"]), rel=1e-15)


def test_nonpositive_pressure_is_ignored(tmp_path):
    """A follower pressure <= 0 adds no constraint (ExternalConstraint.cpp:195-197)."""
    path = golden_files("case_C3D4_nh_pressure.npz")[0]
    from conftest import case_from_golden
    case = case_from_golden(path)
    faces = case.pressure[0][1]
    case.pressure = []
    o_none = oracle.Oracle(oracle.read_case(case.write(str(tmp_path / "none"))))
    case.pressure = [(-5.0, faces)]
    o_neg = oracle.Oracle(oracle.read_case(case.write(str(tmp_path / "neg"))))
    u = np.full(o_none.n_dof, 1e-4)
    assert np.array_equal(o_neg.residual(u), o_none.residual(u))


GRAVITY = golden_files("gravity_*.npz")


@pytest.mark.parametrize("path", GRAVITY, ids=lambda p: p.split("/")[-1][8:-4])
@pytest.mark.parametrize("integration", ["full", "reduced"])
def test_gravity_residual_matches_reference(path, integration, tmp_path):
    """R(u) with the inertia constraint's -M g (consistent or lumped M)."""
    cfg, d = write_golden_case(path, tmp_path, integration)
    case = oracle.read_case(cfg)
    assert case["gravity"] == (0.0, 0.0, -9.8)
    o = oracle.Oracle(case)
    ref = d[f"r_{integration}"]
    assert np.linalg.norm(o.residual(d["u"]) - ref) <= 1e-12 * np.linalg.norm(ref)
    r0 = o.residual(np.zeros(o.n_dof))
    assert np.linalg.norm(r0 - d["r_zero"]) <= 1e-12 * np.linalg.norm(d["r_zero"])


@pytest.mark.parametrize("path", GRAVITY, ids=lambda p: p.split("/")[-1][8:-4])
def test_gravity_solve_matches_reference(path, tmp_path):
    cfg, d = write_golden_case(path, tmp_path)
    o = oracle.Oracle(oracle.read_case(cfg))
    u, info = o.solve()
    ref = d["u_solve"]
    assert info["r_inf"] <= 1e-6
    assert np.linalg.norm(u - ref) <= 1e-6 * np.linalg.norm(ref)
    assert abs(info["niter"] - json.loads(str(d["solve_meta"]))["niter"]) <= 2


def test_gravity_mass_totals(tmp_path):
    """Summed over a body with no fixed nodes, M g gives the weight
    rho g sum_e V_e for either mass (the Gauss weights of each element sum to
    one).  V_e is the reference's corner-face volume, which warped hexahedra
    make differ slightly from the box's L W H."""
    path = golden_files("gravity_C3D8_consistent.npz")[0]
    cfg, d = write_golden_case(path, tmp_path)
    case = oracle.read_case(cfg)
    case["fixed"][:] = 0
    case["forces"] = []
    vol = 0.03 * 0.01 * 0.01
    totals = []
    for consistent in (True, False):
        case["consistent_inertia"] = consistent
        o = oracle.Oracle(case)
        f = -o.residual(np.zeros(o.n_dof)).reshape(-1, 3).sum(axis=0)
        assert np.allclose(f, [0.0, 0.0, -9.8 * 2.0e5 * vol], rtol=1e-4, atol=1e-12)
        totals.append(f)
    assert np.allclose(totals[0], totals[1], rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("key", list(np.load(golden_files("traces.npz")[0]).files))
def test_trace_matches_reference(key, tmp_path):
    """The restatement's convergence record against the reference's benchmark
    vector (||r||_2 after the initial residual and after each line search).
    Rounding differences grow along the iteration path, so the early records
    agree tightly and the whole record to 1e-5 of the initial norm."""
    from efem_b200 import meshgen as mg
    ref = np.load(golden_files("traces.npz")[0])[key]
    et, mat, load = key.split("_")
    o = oracle.Oracle(oracle.read_case(mg.small_case(et, mat, load).write(str(tmp_path))))
    _, info = o.solve(trace=1000)
    t = info["trace"]
    assert len(t) == info["niter"] + 1 and abs(len(t) - len(ref)) <= 2
    assert t[0, 3] == 0.0 and np.all(t[1:, 3] != 0.0) and int(t[:, 4].sum()) == info["r_evals"]
    k = min(len(t), len(ref))
    rel = np.abs(t[:k, 1] - ref[:k]) / ref[:k]
    assert rel[:20].max() <= 1e-8 and rel[:50].max() <= 1e-6
    assert np.abs(t[:k, 1] - ref[:k]).max() <= 1e-5 * ref[0]
