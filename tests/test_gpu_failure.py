"""Failure paths of the solve, each caused on the host or by a bounded
device wait -- none faults, traps or hangs the GPU.

* Singular approximate Jacobian: a free node that no element uses gives the
  scalar matrix L a zero row, so the factorisation meets a zero pivot and
  the solve falls back to H0 = I/theta with EFEM_SOLVE_PRECOND_FALLBACK set,
  as LBFGSSolver::updateApproxJacobi does (src/simulation/nlsolver/LBFGS.h:65-81).
  The fixture failure_orphan_node.npz holds the reference's own fallback
  solve of the same input (tests/golden/make_golden.py failure).
* Non-finite result: a start vector with a NaN gives EFEM_ERR_NAN and the
  solution is zeroed, as Integrator::integral does (src/simulation/Integrator.cpp:28-34).
* A device wait that runs out: options.wait_test makes one wait of each H0
  application wait for a count that no work item produces, and
  options.wait_limit bounds it to a few hundred polls.  The call returns
  EFEM_ERR_TIMEOUT, the output holds NaN, and the next call with the test
  aid off succeeds with the right result in the same CUDA context.
"""
import ctypes
import json

import numpy as np
import pytest

from conftest import golden_files, write_golden_case
from efem_b200 import api

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_singular_jacobian_falls_back_like_the_reference(tmp_path):
    path = golden_files("failure_orphan_node.npz")[0]
    cfg, d = write_golden_case(path, tmp_path)
    meta = json.loads(str(d["solve_meta"]))
    assert meta["precond_ok"] == 0  # the reference took its fallback too
    m = api.Model.from_json(cfg)
    u, info = m.solve()
    assert info["flags"] & api.SOLVE_PRECOND_FALLBACK, info
    assert info["flags"] & api.SOLVE_CONVERGED and info["r_inf"] <= 1e-6, info
    orphan = int(d["orphan_dof"])
    assert np.all(u[orphan:orphan + 3] == 0.0)
    # identity-H0 solves are ill-conditioned: compare converged to 1e-10 N
    m.set_options(residual_criterion=1e-10, max_iterations=50000)
    ut, info = m.solve()
    assert info["flags"] & api.SOLVE_PRECOND_FALLBACK and info["flags"] & api.SOLVE_CONVERGED, info
    assert rel(ut, d["u_tight"]) <= 1e-6, rel(ut, d["u_tight"])


def test_nonfinite_start_returns_nan_status_and_zeroes_u(tmp_path):
    cfg, d = write_golden_case(golden_files("case_C3D8_nh_pressure.npz")[0], tmp_path)
    m = api.Model.from_json(cfg)
    u0 = np.zeros(m.n_dof)
    u0[5] = np.nan
    info = api.SolveInfo()
    st = api.lib().efem_solve(m.h, api._ptr(u0), ctypes.byref(info))
    assert st == api.ERR_NAN, (st, api.last_error())
    assert np.all(u0 == 0.0)
    u, info2 = m.solve()  # the model stays usable
    assert info2["flags"] & api.SOLVE_CONVERGED


def test_wait_that_runs_out_reports_timeout_and_the_gpu_stays_usable(tmp_path):
    cfg, d = write_golden_case(golden_files("case_C3D20_nh_pressure.npz")[0], tmp_path)
    m = api.Model.from_json(cfg)
    v = d["v"]
    good = m.precond_apply(v)  # factors, then one regular H0 application
    m.set_options(wait_test=1, wait_limit=200)
    out = np.array(v)
    st = api.lib().efem_precond_apply(m.h, api._ptr(out))
    assert st == api.ERR_TIMEOUT, (st, api.last_error())
    assert "gave up" in api.last_error()
    assert np.all(np.isnan(out))
    with pytest.raises(api.EfemError) as e:
        m.solve()
    assert e.value.status == api.ERR_TIMEOUT
    m.set_options(wait_test=0, wait_limit=0)
    again = m.precond_apply(v)
    assert rel(again, good) <= 1e-14
    u, info = m.solve()
    assert info["flags"] & api.SOLVE_CONVERGED and info["r_inf"] <= 1e-6
    assert rel(u, d["u_solve"]) <= 1e-6, rel(u, d["u_solve"])
