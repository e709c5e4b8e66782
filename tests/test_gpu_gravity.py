"""Gravity loads (the reference's inertia constraint, -M g in the residual,
src/fe/InertiaConstraint.cpp:34-84) through the CUDA residual and solve,
against the reference's outputs in the gravity fixtures and the oracle."""
import numpy as np
import pytest

import oracle
from conftest import golden_files, write_golden_case
from efem_b200 import api

pytestmark = pytest.mark.gpu
CASES = golden_files("gravity_*.npz")
IDS = lambda p: p.split("/")[-1][8:-4]  # noqa: E731


@pytest.mark.parametrize("path", CASES, ids=IDS)
@pytest.mark.parametrize("integration", ["full", "reduced"])
def test_gravity_residual_fp64_matches_reference(path, integration, tmp_path):
    cfg, d = write_golden_case(path, tmp_path, integration)
    m = api.Model.from_json(cfg)
    ref = d[f"r_{integration}"]
    assert np.linalg.norm(m.residual(d["u"]) - ref) <= 1e-12 * np.linalg.norm(ref)
    r0 = m.residual(np.zeros(m.n_dof))
    assert np.linalg.norm(r0 - d["r_zero"]) <= 1e-11 * np.linalg.norm(d["r_zero"])


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_gravity_residual_mixed_close_to_reference(path, tmp_path):
    cfg, d = write_golden_case(path, tmp_path)
    m = api.Model.from_json(cfg)
    m.set_options(precision=api.MIXED)
    ref = d["r_full"]
    assert np.linalg.norm(m.residual(d["u"]) - ref) <= 2e-5 * np.linalg.norm(ref)


@pytest.mark.parametrize("path", CASES, ids=IDS)
def test_gravity_solve_matches_reference(path, tmp_path):
    """lbfgs_ah at the reference's residual 1e-6 against the reference's solve."""
    cfg, d = write_golden_case(path, tmp_path)
    m = api.Model.from_json(cfg)
    u, info = m.solve()
    assert info["flags"] & api.SOLVE_CONVERGED and info["r_inf"] <= 1e-6
    ref = d["u_solve"]
    assert np.linalg.norm(u - ref) <= 1e-6 * np.linalg.norm(ref)


@pytest.mark.parametrize("path", CASES[::2], ids=IDS)
def test_gravity_tight_solve_matches_oracle(path, tmp_path):
    cfg, _ = write_golden_case(path, tmp_path, residual_criterion=1e-10, max_solver_iters=20000)
    m = api.Model.from_json(cfg)
    u, info = m.solve()
    assert info["flags"] & api.SOLVE_CONVERGED
    uo, _ = oracle.Oracle(oracle.read_case(cfg)).solve()
    assert np.linalg.norm(u - uo) <= 1e-7 * np.linalg.norm(uo)


def test_gravity_mass_switch_reaches_the_device(tmp_path):
    """consistent_inertia changed after a solve: the captured graphs see the
    new M g (same device buffer, new values)."""
    lumped = golden_files("gravity_C3D8_lumped.npz")[0]
    dc = np.load(golden_files("gravity_C3D8_consistent.npz")[0])
    cfg, dl = write_golden_case(lumped, tmp_path)
    m = api.Model.from_json(cfg)
    u, _ = m.solve()
    assert np.linalg.norm(u - dl["u_solve"]) <= 1e-6 * np.linalg.norm(dl["u_solve"])
    m.set_options(consistent_inertia=1)
    assert np.linalg.norm(m.residual(dc["u"]) - dc["r_full"]) <= 1e-12 * np.linalg.norm(dc["r_full"])
    u, _ = m.solve()
    assert np.linalg.norm(u - dc["u_solve"]) <= 1e-6 * np.linalg.norm(dc["u_solve"])
