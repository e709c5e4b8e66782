"""The factor on full-size meshes, by a property that holds at any size:
H0 = (L (x) I3)^{-1}, so (L (x) I3) H0 v = v, with L the approximate
Jacobian the library hands out on the host (efem_approx_jacobian_csr, pinned
to the reference's triplets in test_host.py).  These meshes have panel steps
with more CTAs than one wave of the GPU, and fronts whose rows below the
diagonal block span several CTAs."""
import numpy as np
import pytest

from efem_b200 import api, meshgen as mg

pytestmark = pytest.mark.gpu


def l_times(m, x):
    """(L (x) I3) x on the host from the library's CSR of L."""
    rp, ci, v = m.approx_jacobian_csr()
    X = x.reshape(-1, 3)
    rows = np.repeat(np.arange(m.n_free), np.diff(rp))
    out = np.zeros_like(X)
    np.add.at(out, rows, v[:, None] * X[ci])
    return out.ravel()


@pytest.mark.parametrize("name", ["cap", "finger", "beam"])
def test_factor_inverts_the_approximate_jacobian(name):
    if name == "cap":
        case = mg.cylinder_cap_c3d20()
    elif name == "finger":
        case, _ = mg.finger_c3d10()
    else:
        case = mg.cantilever_c3d8_force()
    m = api.Model.from_case(case)
    v = np.random.default_rng(12).standard_normal(m.n_dof)
    hv = m.precond_apply(v)  # raises if the factor is not positive definite
    back = l_times(m, hv)
    assert np.linalg.norm(back - v) <= 1e-9 * np.linalg.norm(v)
    # and the solve uses it (no fallback to H0 = I / theta).  The beam's solve
    # does not converge, in the reference either (its record is pinned in
    # test_gpu_reference_problems.py): only its first iterations are run.
    m.set_options(max_iterations=6 if name == "beam" else 3000)
    _, info = m.solve()
    assert not info["flags"] & api.SOLVE_PRECOND_FALLBACK, info
    assert name == "beam" or info["flags"] & api.SOLVE_CONVERGED, info
