"""Deterministic scatter (options.deterministic = 1): element and face nodal
forces go to their own slots and each node sums them in a fixed order, so
residuals, solves and batched solves are bitwise repeatable; values agree with
the atomic scatter to rounding and with the reference's outputs."""
import numpy as np
import pytest

from conftest import golden_files, write_golden_case
from efem_b200 import api, meshgen as mg

pytestmark = pytest.mark.gpu
CASES = golden_files()[::4] + golden_files("gravity_C3D20_*.npz")


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.split("/")[-1][:-4])
@pytest.mark.parametrize("precision", [api.FP64, api.MIXED])
def test_residual_deterministic(path, precision, tmp_path):
    cfg, d = write_golden_case(path, tmp_path)
    m = api.Model.from_json(cfg)
    m.set_options(precision=precision)
    r_atomic = m.residual(d["u"])
    m.set_options(deterministic=1)
    r1 = m.residual(d["u"])
    r2 = m.residual(d["u"])
    assert np.array_equal(r1, r2)
    tol = 1e-13 if precision == api.FP64 else 1e-6
    assert np.linalg.norm(r1 - r_atomic) <= tol * np.linalg.norm(r_atomic)
    if precision == api.FP64:
        ref = d["r_full"]
        assert np.linalg.norm(r1 - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.split("/")[-1][:-4])
def test_solve_bitwise_repeatable(path, tmp_path):
    cfg, d = write_golden_case(path, tmp_path)
    m = api.Model.from_json(cfg)
    m.set_options(deterministic=1, trace=1000)
    u1, i1 = m.solve()
    t1 = m.solve_trace()
    u2, i2 = m.solve()
    t2 = m.solve_trace()
    assert np.array_equal(u1, u2) and i1["niter"] == i2["niter"]
    assert np.array_equal(t1["r_norm2"], t2["r_norm2"])
    assert i1["flags"] & api.SOLVE_CONVERGED
    ref = d["u_solve"]
    assert np.linalg.norm(u1 - ref) <= 1e-6 * np.linalg.norm(ref)
    # the host-driven loop runs the same kernels in the same order
    m.set_options(host_loop=1)
    u3, i3 = m.solve()
    assert np.array_equal(u1, u3) and i3["niter"] == i1["niter"]


def test_batch_equals_single_solves_bitwise():
    cases = mg.batch_beams(n=4, seed=11, el_min=500, el_max=2000)

    def models():
        out = []
        for c in cases:
            m = api.Model.from_case(c)
            m.set_options(deterministic=1)
            out.append(m)
        return out

    single = [m.solve()[0] for m in models()]
    us, infos = api.batch_solve(models(), max_threads=4)
    for u, ref, info in zip(us, single, infos):
        assert info["flags"] & api.SOLVE_CONVERGED
        assert np.array_equal(u, ref)
