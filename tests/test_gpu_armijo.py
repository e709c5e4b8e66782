"""The Armijo line search (options.line_search = 1): steps halve from 1 until
the total potential Pi(u) = E(u) - f_ext.u (FP64 strain-energy sum) falls by
at least 1e-4 a r.d.  It solves the same equilibria as the reference's
residual-projection rule, for conservative loads (nodal forces, gravity)."""
import numpy as np
import pytest

from conftest import golden_files, write_golden_case
from efem_b200 import api, meshgen as mg

pytestmark = pytest.mark.gpu
CASES = golden_files("case_*_force.npz")[::3] + golden_files("gravity_*_consistent.npz")[::2]


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.split("/")[-1][:-4])
def test_armijo_solves_the_same_equilibrium(path, tmp_path):
    cfg, d = write_golden_case(path, tmp_path, residual_criterion=1e-10, max_solver_iters=20000)
    ref = api.Model.from_json(cfg)
    u_ref, i_ref = ref.solve()
    m = api.Model.from_json(cfg)
    m.set_options(line_search=1, trace=20000)
    u, info = m.solve()
    assert info["flags"] & api.SOLVE_CONVERGED, info
    assert np.linalg.norm(u - u_ref) <= 1e-7 * np.linalg.norm(u_ref)
    # at the reference's tolerance, against the reference's own solve
    assert np.linalg.norm(u - d["u_solve"]) <= 1e-5 * np.linalg.norm(d["u_solve"])
    # the accepted steps are 1, 1/2, 1/4, ... (the reference rule also grows steps by 1.5)
    steps = m.solve_trace()["step"][1:]
    assert len(steps) == info["niter"]
    assert np.all(steps <= 1.0) and np.all(np.abs(np.log2(steps) - np.round(np.log2(steps))) < 1e-12)
    # Pi decreased from u = 0
    assert m.strain_energy(u) - float(m.external_load() @ u) < 0.0


def test_armijo_energy_decreases_every_iteration():
    case = mg.small_case("C3D8", "mr", "force")
    m = api.Model.from_case(case)
    pis = []
    u = np.zeros(m.n_dof)
    for it in range(1, 40):
        m.set_options(line_search=1, max_iterations=it)
        u_it, _ = m.solve(np.zeros(m.n_dof))
        pis.append(m.strain_energy(u_it) - float(m.external_load() @ u_it))
    assert all(b <= a + 1e-15 * abs(a) for a, b in zip(pis, pis[1:])), pis


def test_armijo_refuses_pressure_loads():
    m = api.Model.from_case(mg.small_case("C3D4", "nh", "pressure"))
    m.set_options(line_search=1)
    with pytest.raises(api.EfemError, match="conservative"):
        m.solve()
