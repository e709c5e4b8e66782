"""Converged displacements against the reference on its own sample problems,
on the large benchmark meshes and on a multi-body case.

Fixtures (tests/golden/make_golden.py, the reference compiled from its
sources by oracle/Makefile):

* ``sample_<problem>_<variant>.npz`` -- the reference's six sample problems
  (beam C3D4 / C3D20 under directed pressure with the ``id: -1``
  Mooney-Rivlin material, cap C3D4 / C3D20 and finger C3D4 / C3D10 under
  follower pressure), their own JSON configs (``max_optim_iters``) and files,
  with the reference's solution at the config's tolerance (``u_solve``,
  ||r||_inf <= 1e-6 N) and at 1e-10 N (``u_tight``);
* ``config_<name>.npz`` -- the reference's solution of the generated C3D20R
  cylinder cap and C3D10 Yeoh finger at 1e-6 N;
* ``config_beam_c3d8_mr_force_record.npz`` -- the reference's benchmark record
  of the generated C3D8 Mooney-Rivlin beam (80x16x16, tip forces), whose
  solve does not converge;
* ``multibody_c3d10_pose.npz`` -- two posed bodies with per-element material
  ids and model_id-routed constraints: R(u) at a seeded u and the solution.

The reference path is LBFGSSolver::solve (src/simulation/nlsolver/LBFGS.h:96-174).
Two solves that stop inside the same ||r||_inf <= eps ball differ by up to
the ball's size in displacement, so the FP64 solution is compared with the
reference at 1e-10 N to 1e-6 relative L2, and the solution at the
reference's own 1e-6 N criterion is held to ten times the distance the
reference's own solve keeps there from its 1e-10 N solution, with a floor of
1e-6.  The mixed-precision path (FP32 element kernels) is held to 1e-4.
"""
import json

import numpy as np
import pytest

from conftest import GOLDEN, golden_files, write_sample
from efem_b200 import api

pytestmark = pytest.mark.gpu
SAMPLES = golden_files("sample_*.npz")


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("path", SAMPLES, ids=lambda p: p.split("/")[-1][7:-4])
def test_sample_fp64_matches_reference(path, tmp_path):
    cfg, d = write_sample(path, tmp_path)
    m = api.Model.from_json(cfg)
    u, info = m.solve()
    assert info["flags"] & api.SOLVE_CONVERGED and not info["flags"] & api.SOLVE_PRECOND_FALLBACK, info
    assert info["r_inf"] <= 1e-6
    ref_t, ref = d["u_tight"], d["u_solve"]
    # how far the reference's own 1e-6 N solve is from equilibrium: one sample
    # of where a solve stops inside the tolerance ball; the GPU's stopping
    # point (its atomic scatter changes the rounding, hence the path) is held
    # to ten times that, with a floor of 1e-6
    own = rel(ref, ref_t)
    assert rel(u, ref_t) <= max(1e-6, 10.0 * own), (rel(u, ref_t), own, info["niter"])
    m.set_options(residual_criterion=1e-10, max_iterations=20000)
    ut, info = m.solve()
    assert info["flags"] & api.SOLVE_CONVERGED, info
    assert rel(ut, ref_t) <= 1e-6, rel(ut, ref_t)


@pytest.mark.parametrize("path", SAMPLES, ids=lambda p: p.split("/")[-1][7:-4])
def test_sample_mixed_matches_reference(path, tmp_path):
    """FP32 element kernels (FP64 factor, norms and L-BFGS vectors): within
    1e-4 relative L2 of the reference's equilibrium."""
    cfg, d = write_sample(path, tmp_path)
    m = api.Model.from_json(cfg)
    m.set_options(precision=api.MIXED)
    u, info = m.solve()
    assert info["flags"] & api.SOLVE_CONVERGED, info
    assert rel(u, d["u_tight"]) <= 1e-4, rel(u, d["u_tight"])


def test_multibody_pose_model_id_matches_reference(tmp_path):
    path = golden_files("multibody_c3d10_pose.npz")[0]
    cfg, d = write_sample(path, tmp_path)
    m = api.Model.from_json(cfg)
    assert m.n_dof == d["u"].shape[0]
    r = m.residual(d["u"])
    assert rel(r, d["r"]) <= 1e-12, rel(r, d["r"])
    u, info = m.solve()
    assert info["flags"] & api.SOLVE_CONVERGED and info["r_inf"] <= 1e-8, info
    assert rel(u, d["u_solve"]) <= 1e-6, rel(u, d["u_solve"])


def _config(name):
    import sys
    import os
    sys.path.insert(0, os.path.dirname(GOLDEN))
    from golden.make_golden import config_case, mesh_digest
    path = golden_files(f"config_{name}.npz")
    if not path:
        pytest.skip(f"no fixture for {name}")
    d = np.load(path[0], allow_pickle=False)
    case, reduced = config_case(name)
    assert mesh_digest(case) == str(d["mesh"]), "the generator no longer makes the fixture's mesh"
    case.integration = "reduced" if reduced else "full"
    return case, d


def test_config_beam_follows_the_reference_record():
    """The C3D8 Mooney-Rivlin beam under 0.5 N tip forces: the reference's own
    solve does not converge -- at its seventh iteration the line search
    accepts a trial with elements turned inside out, and ||r|| passes 1e9 N
    two iterations later.  ||r||_2 after the initial residual and each line
    search, against the reference's record: records 0-7 to 1e-6 relative,
    then the same blow-up (every later record above 1e8 N in both)."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(GOLDEN))
    from golden.make_golden import config_case, mesh_digest
    d = np.load(golden_files("config_beam_c3d8_mr_force_record.npz")[0], allow_pickle=False)
    case, _ = config_case("beam_c3d8_mr_force")
    assert mesh_digest(case) == str(d["mesh"]), "the generator no longer makes the fixture's mesh"
    ref = d["r_norm2"]
    n = len(ref)
    m = api.Model.from_case(case)
    m.set_options(trace=n, max_iterations=n - 1)
    u = np.zeros(m.n_dof)
    st = api.lib().efem_solve(m.h, api._vec_ptr(u), None)
    # past the eighth line search the path follows rounding; a solve may even
    # end non-finite there (EFEM_ERR_NAN), as the reference's may
    assert st in (api.OK, api.ERR_NAN), api.last_error()
    tr = m.solve_trace()["r_norm2"]
    assert len(tr) >= 9, len(tr)
    rel = np.abs(tr[:8] - ref[:8]) / ref[:8]
    assert rel.max() <= 1e-6, rel
    k = min(len(tr), n)
    assert np.all(~np.isfinite(tr[8:k]) | (tr[8:k] > 1e6)) and ref[8:].min() > 1e8, (tr, ref)


@pytest.mark.parametrize("name", ["cap_c3d20r_nh_pressure", "finger_c3d10_yeoh_pressure"])
def test_config_fp64_matches_reference(name):
    """FP64 solve of the large benchmark meshes at the reference's 1e-6 N
    criterion against the reference's own solve at the same criterion."""
    case, d = _config(name)
    m = api.Model.from_case(case)
    m.set_options(residual_criterion=float(d["epsilon"]))
    u, info = m.solve()
    assert info["flags"] & api.SOLVE_CONVERGED and not info["flags"] & api.SOLVE_PRECOND_FALLBACK, info
    err = rel(u, d["u_solve"].astype(np.float64))
    meta = json.loads(str(d["solve_meta"]))
    assert err <= 1e-6, (err, info["niter"], meta["niter"])
