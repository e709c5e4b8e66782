"""True tangent, parameter derivatives and adjoint sensitivities.

The reference has no tangent or adjoint; its residual is the anchor.  The
residual is pinned to the reference (test_gpu_residual.py), and every
derivative here is checked against central finite differences of that
residual, or of re-solved equilibria for the adjoint gradient.
"""
import copy

import numpy as np
import pytest

from efem_b200 import api, meshgen as mg

pytestmark = pytest.mark.gpu

COMBOS = [("C3D4", "nh", "pressure"), ("C3D8", "mr", "dpressure"), ("C3D10", "yeoh", "pressure"),
          ("C3D20", "nh", "force"), ("C3D8", "yeoh", "top_pressure"), ("C3D10", "mr", "dpressure")]


def solved(case, crit=1e-10):
    case = copy.deepcopy(case)
    m = api.Model.from_case(case)
    m.set_options(residual_criterion=crit, max_iterations=20000)
    u, info = m.solve()
    assert info["flags"] & api.SOLVE_CONVERGED, info
    return m, u


@pytest.mark.parametrize("etype,mat,load", COMBOS)
def test_hvp_matches_finite_differences(etype, mat, load):
    """K(u) v against (R(u + h v) - R(u - h v)) / 2h at an equilibrium."""
    m, u = solved(mg.small_case(etype, mat, load))
    rng = np.random.default_rng(3)
    v = rng.standard_normal(m.n_dof) * np.abs(u).max()
    h = 1e-5
    fd = (m.residual(u + h * v) - m.residual(u - h * v)) / (2 * h)
    kv = m.hvp(u, v)
    assert np.linalg.norm(kv - fd) <= 2e-6 * np.linalg.norm(kv)


@pytest.mark.parametrize("etype,mat,load", COMBOS)
def test_hvp_transpose(etype, mat, load):
    """w.(K v) = (K^T w).v; without pressure faces K is symmetric."""
    m, u = solved(mg.small_case(etype, mat, load))
    rng = np.random.default_rng(4)
    v, w = rng.standard_normal(m.n_dof), rng.standard_normal(m.n_dof)
    kv, ktw = m.hvp(u, v), m.hvp(u, w, transpose=True)
    lhs, rhs = float(w @ kv), float(ktw @ v)
    assert abs(lhs - rhs) <= 1e-11 * np.linalg.norm(kv) * np.linalg.norm(w)
    if load == "force":
        assert np.linalg.norm(m.hvp(u, v, transpose=True) - kv) <= 1e-11 * np.linalg.norm(kv)


def perturbed(case, k, h):
    """The case with parameter k (efem_residual_param_derivative order) moved by h."""
    c = copy.deepcopy(case)
    names = ["C10", "C01", "C20", "C30", "D1"]
    if k < 5 * len(c.materials):
        c.materials[k // 5][names[k % 5]] = c.materials[k // 5].get(names[k % 5], 0.0) + h
    else:
        value, faces = c.pressure[k - 5 * len(c.materials)]
        if isinstance(value, (list, tuple, np.ndarray)):
            value = list(np.asarray(value, dtype=float) * (1.0 + h))  # the scale of a directed load moves by h
        else:
            value = value + h
        c.pressure[k - 5 * len(c.materials)] = (value, faces)
    return c


def scale_of(case, k):
    names = ["C10", "C01", "C20", "C30", "D1"]
    if k < 5 * len(case.materials):
        val = case.materials[k // 5].get(names[k % 5], 0.0)
        return abs(val) if val != 0 else 1e4
    value, _ = case.pressure[k - 5 * len(case.materials)]
    return abs(value) if not isinstance(value, (list, tuple, np.ndarray)) else 1.0


@pytest.mark.parametrize("etype,mat,load", COMBOS)
def test_param_derivative_matches_finite_differences(etype, mat, load):
    case = mg.small_case(etype, mat, load)
    m, u = solved(case)
    ds, fds = [], []
    for k in range(m.n_params):
        h = 1e-5 * scale_of(case, k)
        rp = api.Model.from_case(perturbed(case, k, h)).residual(u)
        rm = api.Model.from_case(perturbed(case, k, -h)).residual(u)
        fds.append((rp - rm) / (2 * h) * scale_of(case, k))
        ds.append(m.param_derivative(u, k) * scale_of(case, k))
    # derivatives scaled to relative parameter changes; parameters a law does
    # not use (C01 of a Neo-Hookean material) have derivative 0 up to rounding
    top = max(np.linalg.norm(d) for d in ds)
    for k, (d, fd) in enumerate(zip(ds, fds)):
        assert np.linalg.norm(d - fd) <= 2e-6 * max(np.linalg.norm(d), np.linalg.norm(fd)) + 1e-10 * top, \
            (k, np.linalg.norm(d), np.linalg.norm(fd))


@pytest.mark.parametrize("etype,mat,load", [("C3D10", "yeoh", "pressure"), ("C3D8", "mr", "dpressure"),
                                            ("C3D4", "nh", "top_pressure")])
def test_adjoint_gradient_matches_finite_differences(etype, mat, load):
    """J = u_z of the tip node farthest along x; dJ/dtheta by the adjoint
    against central differences of re-solved equilibria (relative step 1e-4)."""
    case = mg.small_case(etype, mat, load)
    m, u = solved(case, 1e-11)
    X = case.mesh.X
    node_of_dof = m.dof_map()
    tip = int(np.argmax(X[node_of_dof, 0] + 1e-3 * X[node_of_dof, 2]))
    dof = 3 * tip + 2
    g = np.zeros(m.n_dof)
    g[dof] = 1.0
    m.set_options(adjoint_tolerance=1e-10)
    grad, lam, info = m.adjoint(u, g, want_lambda=True)
    assert info["flags"] & api.SOLVE_CONVERGED, info
    # every Krylov iteration launches kernels and moves at least the basis
    # vector and one H0 application's factor entries
    assert info["n_kernel_launches"] >= 5 * info["iterations"]
    assert info["solve_bytes"] >= info["iterations"] * 16.0 * m.info()["factor_nnz"]
    # the adjoint equation holds (the stored tangents of the solve against the
    # dual-number transpose product)
    assert np.linalg.norm(m.hvp(u, lam, transpose=True) - g) <= 1e-8
    fds = []
    for k in range(m.n_params):
        val = scale_of(case, k)
        h = 1e-4 * val
        Js = []
        for sgn in (1, -1):
            mk = api.Model.from_case(perturbed(case, k, sgn * h))
            mk.set_options(residual_criterion=1e-11, max_iterations=20000)
            uk, ik = mk.solve(u.copy())
            assert ik["flags"] & api.SOLVE_CONVERGED
            Js.append(uk[dof])
        fd = (Js[0] - Js[1]) / (2 * h)
        fds.append(fd)
    # compare sensitivities to relative parameter changes, theta_k dJ/dtheta_k
    sc = np.array([scale_of(case, k) for k in range(m.n_params)])
    a, b = grad * sc, np.array(fds) * sc
    assert np.all(np.abs(a - b) <= 1e-3 * np.abs(a).max() + 2e-4 * np.abs(b)), (a, b)


def test_adjoint_device_pointers_match_host():
    import torch
    case = mg.small_case("C3D10", "yeoh", "pressure")
    m, u = solved(case)
    g = np.random.default_rng(5).standard_normal(m.n_dof)
    grad_h, lam_h, _ = m.adjoint(u, g, want_lambda=True)
    m.set_options(device_ptrs=1)
    ut, gt = torch.tensor(u, device="cuda"), torch.tensor(g, device="cuda")
    grad_d, lam_d, _ = m.adjoint(ut, gt, want_lambda=True)
    assert np.allclose(grad_d, grad_h, rtol=1e-9, atol=0)
    assert np.allclose(lam_d.cpu().numpy(), lam_h, rtol=1e-9, atol=1e-12 * np.abs(lam_h).max())


@pytest.mark.parametrize("etype,mat", [("C3D4", "nh"), ("C3D8", "mr"), ("C3D10", "yeoh"), ("C3D20", "mr")])
def test_strain_energy_gradient_is_internal_force(etype, mat):
    """dE/du . v by central differences equals f_int(u) . v, f_int = R(u) - R(0)
    for a case with nodal forces only; E(0) = 0."""
    case = mg.small_case(etype, mat, "force")
    m, u = solved(case)
    assert m.strain_energy(np.zeros(m.n_dof)) == 0.0
    rng = np.random.default_rng(6)
    v = rng.standard_normal(m.n_dof) * np.abs(u).max()
    # the nearly incompressible penalty (D1 = 1e-6) makes the third derivative
    # large along a random direction: the central difference needs a small step
    # (its error falls as h^2: 6e-5 relative at h = 1e-4, 7e-9 at 1e-6 on C3D4)
    h = 1e-7
    fd = (m.strain_energy(u + h * v) - m.strain_energy(u - h * v)) / (2 * h)
    fint = m.residual(u) - m.residual(np.zeros(m.n_dof))
    assert abs(fd - float(fint @ v)) <= 1e-5 * abs(float(fint @ v))
    assert m.strain_energy(u) > 0


@pytest.mark.parametrize("etype,mat,load", [("C3D10", "yeoh", "pressure"), ("C3D8", "mr", "dpressure")])
def test_adjoint_without_stored_tangents_matches(etype, mat, load, monkeypatch):
    """When the stored tangents cannot be allocated (forced here with
    EFEM_TEST_STORED_OOM=1, which makes their allocation report out of
    memory) the adjoint falls back to dual-number products: same gradient,
    a successful call and no stale allocation error text."""
    case = mg.small_case(etype, mat, load)
    m, u = solved(case)
    g = np.zeros(m.n_dof)
    g[-1] = 1.0
    want, _, info = m.adjoint(u, g)
    m2, _ = solved(case)
    monkeypatch.setenv("EFEM_TEST_STORED_OOM", "1")
    got, _, info2 = m2.adjoint(u, g)
    assert info2["flags"] & api.SOLVE_CONVERGED, info2
    assert np.linalg.norm(got - want) <= 1e-8 * np.linalg.norm(want)
    assert "cudaMalloc" not in api.last_error(), api.last_error()
