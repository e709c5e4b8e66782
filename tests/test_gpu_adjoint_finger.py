"""The adjoint gradient at the size of the benchmark's finger (50 688 C3D10
Yeoh elements, 240 600 DOF, 30 kPa on the chamber walls): dJ/dtheta of
J = u_z of the tip node against central finite differences of equilibria
re-solved on the GPU (relative step 1e-4, as the benchmark specifies), for
C10, C20 and the pressure, to 1e-5 relative (north_star's target).  The
reference has no tangent or adjoint; the residual these derivatives come
from is pinned to it (test_gpu_residual.py, and the finger's solution to the
reference's own solve in test_gpu_reference_problems.py)."""
import copy

import numpy as np
import pytest

from efem_b200 import api, meshgen as mg

pytestmark = pytest.mark.gpu
TIGHT = 1e-11


def solve(case, u0=None):
    m = api.Model.from_case(case)
    m.set_options(residual_criterion=TIGHT, max_iterations=50000, deterministic=1, adjoint_tolerance=1e-11)
    u, info = m.solve(None if u0 is None else np.array(u0))
    assert info["flags"] & api.SOLVE_CONVERGED, info
    return m, u


def test_finger_adjoint_matches_central_differences():
    case, tip = mg.finger_c3d10()
    m, u = solve(case)
    dnode = int(np.nonzero(m.dof_map() == tip)[0][0])
    dof = 3 * dnode + 2
    g = np.zeros(m.n_dof)
    g[dof] = 1.0
    grad, _, info = m.adjoint(u, g)
    assert info["flags"] & api.SOLVE_CONVERGED, info
    # parameter order: 5 per material slot (C10, C01, C20, C30, D1), then each pressure load
    checks = {0: ("C10", None), 2: ("C20", None), 5: (None, "pressure")}
    for k, (name, load) in checks.items():
        c_plus, c_minus = copy.deepcopy(case), copy.deepcopy(case)
        if name:
            th = case.materials[0][name]
            h = 1e-4 * abs(th)
            c_plus.materials[0][name] = th + h
            c_minus.materials[0][name] = th - h
        else:
            p0, faces = case.pressure[0]
            h = 1e-4 * abs(p0)
            c_plus.pressure[0] = (p0 + h, faces)
            c_minus.pressure[0] = (p0 - h, faces)
        up = solve(c_plus, u)[1][dof]
        um = solve(c_minus, u)[1][dof]
        fd = (up - um) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-5 * abs(fd), (k, grad[k], fd)
