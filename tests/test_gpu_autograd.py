"""The adjoint behind a torch.autograd.Function (test harness only).

``EquilibriumSolve.apply(theta)`` returns the equilibrium displacement u(theta)
of a case whose parameters theta are, in efem_residual_param_derivative order,
(C10, C01, C20, C30, D1) of every material and then the magnitude of every
pressure load (a follower pressure in Pa; the scale of a directed load, 1 at
the case's own vector).  Its backward is one adjoint solve,
dJ/dtheta = -lambda . dR/dtheta with K(u)^T lambda = dJ/du, through the C ABI.

The gradients of J(u(theta)) are checked against central finite differences
with a relative step of 1e-4 of equilibria re-solved on the GPU, and against
the same differences of equilibria solved by the oracle (the FP64 CPU
restatement of the reference's solver, pinned to the reference's outputs):
both to 1e-5 relative.
"""
import copy
import tempfile

import numpy as np
import pytest
import torch

import oracle
from efem_b200 import api, meshgen as mg

pytestmark = pytest.mark.gpu

NAMES = ["C10", "C01", "C20", "C30", "D1"]
# Residual of the re-solved equilibria behind the differences.  The softest
# (bending) mode of these small cantilevers has a stiffness of about 60 N/m,
# so a residual r moves u by about r / 60 m; with a relative step of 1e-4 the
# differences resolve J to 1e-5 only for r below about 1e-12 (at 1e-11 they
# are off by 2e-5).  1e-13 N is well above the FP64 floor of the residual
# (about 5e-14 N here).
TIGHT = 1e-13


def theta_of(case):
    th = [float(mat.get(k, 0.0)) for mat in case.materials for k in NAMES]
    for value, _ in case.pressure:
        th.append(1.0 if isinstance(value, (list, tuple, np.ndarray)) else float(value))
    return np.array(th)


def case_at(case, theta):
    c = copy.deepcopy(case)
    k = 0
    for mat in c.materials:
        for name in NAMES:
            if name in mat or theta[k] != 0.0:
                mat[name] = float(theta[k])
            k += 1
    for i, (value, faces) in enumerate(c.pressure):
        if isinstance(value, (list, tuple, np.ndarray)):
            value = [float(theta[k]) * float(v) for v in value]
        else:
            value = float(theta[k])
        c.pressure[i] = (value, faces)
        k += 1
    return c


def gpu_solve(case, u0=None, crit=TIGHT):
    m = api.Model.from_case(case)
    m.set_options(residual_criterion=crit, max_iterations=20000, deterministic=1, adjoint_tolerance=1e-10)
    u, info = m.solve(None if u0 is None else np.array(u0))
    assert info["flags"] & api.SOLVE_CONVERGED, info
    return m, u


class EquilibriumSolve(torch.autograd.Function):
    """u(theta) by the GPU solve; the backward is the GPU adjoint."""

    @staticmethod
    def forward(ctx, theta, case):
        m, u = gpu_solve(case_at(case, theta.detach().cpu().numpy()))
        ctx.model, ctx.u = m, u
        return torch.from_numpy(u)

    @staticmethod
    def backward(ctx, grad_u):
        g = np.ascontiguousarray(grad_u.detach().cpu().numpy(), dtype=np.float64)
        grad, _, info = ctx.model.adjoint(ctx.u, g)
        assert info["flags"] & api.SOLVE_CONVERGED, info
        return torch.from_numpy(grad), None


def tip_dof(case, m):
    X = case.mesh.X[m.dof_map()]
    return 3 * int(np.argmax(X[:, 0] + 1e-3 * X[:, 2])) + 2


def objectives(u, dof, scale):
    """J1 = u_z of the tip node (the finger's objective); J2 = a smooth
    nonlinear function of every displacement."""
    return u[dof], torch.sum((u / scale) ** 2) * scale


CASES = [("C3D10", "yeoh", "pressure"), ("C3D8", "mr", "dpressure"), ("C3D4", "nh", "top_pressure")]


@pytest.mark.parametrize("etype,mat,load", CASES)
def test_autograd_gradient_matches_finite_differences(etype, mat, load):
    case = mg.small_case(etype, mat, load)
    th0 = theta_of(case)
    theta = torch.tensor(th0, dtype=torch.float64, requires_grad=True)
    u = EquilibriumSolve.apply(theta, case)
    m0, u0 = gpu_solve(case)
    dof, scale = tip_dof(case, m0), float(np.abs(u0).max())
    grads = []
    for J in objectives(u, dof, scale):
        (g,) = torch.autograd.grad(J, theta, retain_graph=True)
        grads.append(g.numpy())

    def J_np(uu):
        t = torch.from_numpy(uu)
        return [float(j) for j in objectives(t, dof, scale)]

    # the parameters the case's law uses (C01 of NH, C20/C30 of MR... give zero rows)
    used = [k for k in range(len(th0)) if th0[k] != 0.0]
    fd_gpu = np.zeros((2, len(th0)))
    fd_orc = np.zeros((2, len(th0)))
    for k in used:
        h = 1e-4 * abs(th0[k])
        Jg, Jo = [], []
        for sgn in (1.0, -1.0):
            th = th0.copy()
            th[k] += sgn * h
            ck = case_at(case, th)
            _, uk = gpu_solve(ck, u0)
            Jg.append(J_np(uk))
            with tempfile.TemporaryDirectory() as td:
                o = oracle.Oracle(oracle.read_case(ck.write(td)))
            uo, io = o.solve(u0=u0, epsilon=TIGHT, max_iterations=20000)
            assert io["r_inf"] <= TIGHT * max(1.0, np.abs(uo).max())
            Jo.append(J_np(uo))
        for j in range(2):
            fd_gpu[j, k] = (Jg[0][j] - Jg[1][j]) / (2 * h)
            fd_orc[j, k] = (Jo[0][j] - Jo[1][j]) / (2 * h)
    for j in range(2):
        # sensitivities to relative parameter changes, theta_k dJ/dtheta_k
        sc = np.where(th0 != 0.0, np.abs(th0), 1.0)
        a, b, c = grads[j][used] * sc[used], fd_gpu[j, used] * sc[used], fd_orc[j, used] * sc[used]
        assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b), (j, a, b)
        assert np.linalg.norm(a - c) <= 1e-5 * np.linalg.norm(c), (j, a, c)
        assert np.all(np.abs(a - b) <= 1e-5 * np.abs(b).max()), (j, a, b)
