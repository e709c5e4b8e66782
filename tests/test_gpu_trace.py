"""The solve's convergence trace (options.trace, efem_solve_trace) against the
reference's benchmark record (src/simulation/nlsolver/LBFGS.h:107-147) in
tests/golden/traces.npz, and its bookkeeping."""
import numpy as np
import pytest

from conftest import golden_files
from efem_b200 import api, meshgen as mg

pytestmark = pytest.mark.gpu
TRACES = np.load(golden_files("traces.npz")[0])


def traced(key, **opts):
    et, mat, load = key.split("_")
    m = api.Model.from_case(mg.small_case(et, mat, load))
    m.set_options(trace=1000, **opts)
    u, info = m.solve()
    return m, u, info, m.solve_trace()


@pytest.mark.parametrize("key", TRACES.files)
def test_trace_matches_reference(key):
    """||r||_2 per iteration: the early records to 1e-7 relative (the
    reductions and the factor's sums are ordered differently from Eigen's),
    the whole record to 1e-4 of the initial norm, and the same number of
    iterations within 3."""
    ref = TRACES[key]
    m, u, info, tr = traced(key)
    t = tr["r_norm2"]
    assert tr["n_records"] == len(t) == info["niter"] + 1
    assert abs(len(t) - len(ref)) <= 3
    k = min(len(t), len(ref))
    rel = np.abs(t[:k] - ref[:k]) / ref[:k]
    assert rel[:20].max() <= 1e-7, rel[:20]
    assert np.abs(t[:k] - ref[:k]).max() <= 1e-4 * ref[0]


@pytest.mark.parametrize("key", TRACES.files[:3])
def test_trace_bookkeeping(key):
    m, u, info, tr = traced(key)
    r0 = m.residual(np.zeros(m.n_dof))
    assert np.isclose(tr["r_norm2"][0], np.linalg.norm(r0), rtol=1e-13)
    assert np.isclose(tr["r_inf"][0], np.abs(r0).max(), rtol=1e-13)
    assert tr["r_inf"][-1] == info["r_inf"]
    assert tr["step"][0] == 0.0 and np.all(tr["step"][1:] != 0.0)
    assert tr["r_evals"].sum() == info["n_residual_evals"] and np.all(tr["r_evals"] >= 1)
    assert np.all(np.diff(tr["time_s"]) >= 0) and tr["time_s"][-1] <= info["ms_total"] * 1e-3
    # the host-driven loop runs the same kernels: the same trace up to the
    # order of the residual's atomic scatter
    m.set_options(host_loop=1)
    _, info2 = m.solve()
    tr2 = m.solve_trace()
    assert abs(info2["niter"] - info["niter"]) <= 3
    assert np.allclose(tr2["r_norm2"][:20], tr["r_norm2"][:20], rtol=1e-9, atol=0)
    assert np.array_equal(tr2["step"][:5], tr["step"][:5])


def test_trace_capacity_and_off():
    key = TRACES.files[0]
    m, u, info, tr = traced(key)
    m.set_options(trace=10)
    m.solve()
    small = m.solve_trace()
    assert abs(small["n_records"] - (info["niter"] + 1)) <= 3 and len(small["r_norm2"]) == 10
    assert np.allclose(small["r_norm2"], tr["r_norm2"][:10], rtol=1e-9, atol=0)
    m.set_options(trace=0)
    m.solve()
    assert len(m.solve_trace()["r_norm2"]) == 0
