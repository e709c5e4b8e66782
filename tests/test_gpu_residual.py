"""CUDA residual R(u) against the reference (golden fixtures) and the oracle.

FP64 element kernels: relative L2 error <= 1e-12.  Mixed path (FP32 element
arithmetic, FP64 accumulation): relative L2 error <= 2e-5 at the fixtures'
random displacements (strain ~1e-3)."""
import numpy as np
import pytest

import oracle
from conftest import golden_files, write_golden_case
from efem_b200 import api, meshgen as mg

pytestmark = pytest.mark.gpu
CASES = golden_files()


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.split("/")[-1][5:-4])
@pytest.mark.parametrize("integration", ["full", "reduced"])
def test_residual_fp64_matches_reference(path, integration, tmp_path):
    cfg, d = write_golden_case(path, tmp_path, integration)
    m = api.Model.from_json(cfg)
    r = m.residual(d["u"])
    ref = d[f"r_{integration}"]
    assert np.linalg.norm(r - ref) <= 1e-12 * np.linalg.norm(ref)
    r0 = m.residual(np.zeros(m.n_dof))
    o = oracle.Oracle(oracle.read_case(cfg))
    ro = o.residual(np.zeros(m.n_dof))
    assert np.abs(r0 - ro).max() <= 1e-9 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.split("/")[-1][5:-4])
def test_residual_mixed_close_to_reference(path, tmp_path):
    cfg, d = write_golden_case(path, tmp_path)
    m = api.Model.from_json(cfg)
    m.set_options(precision=api.MIXED)
    r = m.residual(d["u"])
    ref = d["r_full"]
    assert np.linalg.norm(r - ref) <= 2e-5 * np.linalg.norm(ref)


@pytest.mark.parametrize("path", golden_files("inverted_*.npz"), ids=lambda p: p.split("/")[-1][9:-4])
def test_residual_inverted_elements_match_reference(path, tmp_path):
    """Every element turned inside out (J about -1/2 at every Gauss point):
    the reference's laws take J^{-2/3} as (J^2)^{-1/3} and stay finite, and so
    must R(u) here -- a line search that tries such a state (the C3D8 beam
    under tip forces does) chooses its next step from these values.  FP64 to
    1e-12 relative L2 (both integrations for C3D20), FP32 elements to 1e-4."""
    d0 = np.load(path)
    for integration in (["full", "reduced"] if "r_reduced" in d0.files else ["full"]):
        cfg, d = write_golden_case(path, tmp_path, integration)
        m = api.Model.from_json(cfg)
        r = m.residual(d["u"])
        ref = d[f"r_{integration}"]
        assert np.all(np.isfinite(r))
        assert np.linalg.norm(r - ref) <= 1e-12 * np.linalg.norm(ref), (integration, np.linalg.norm(r - ref))
        m.set_options(precision=api.MIXED)
        rm = m.residual(d["u"])
        assert np.linalg.norm(rm - ref) <= 1e-4 * np.linalg.norm(ref), (integration, np.linalg.norm(rm - ref))


def test_residual_device_pointers():
    import torch
    case = mg.cantilever_c3d4_pressure()
    m = api.Model.from_case(case)
    u = np.random.default_rng(3).normal(size=m.n_dof) * 1e-4
    r_host = m.residual(u)
    m.set_options(device_ptrs=1)
    ut = torch.tensor(u, device="cuda", dtype=torch.float64)
    rt = torch.zeros_like(ut)
    m.residual(ut, rt)
    torch.cuda.synchronize()
    assert np.array_equal(rt.cpu().numpy(), r_host) or np.allclose(rt.cpu().numpy(), r_host, rtol=1e-13, atol=1e-15)


def test_residual_large_mesh_against_oracle():
    """Size-independent check on the 20 480-element C3D8 beam: the residual at a
    smooth displacement field matches the oracle to 1e-12 (relative L2)."""
    case = mg.cantilever_c3d8_force(nx=40, ny=8, nz=8)
    m = api.Model.from_case(case)
    X = case.mesh.X[m.dof_map()]
    u = (1e-3 * np.stack([np.sin(30 * X[:, 0]), X[:, 0] * X[:, 1], np.cos(20 * X[:, 2])], axis=1)).ravel()
    r = m.residual(u)
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        o = oracle.Oracle(oracle.read_case(case.write(td)))
        ro = o.residual(u)
    assert np.linalg.norm(r - ro) <= 1e-12 * np.linalg.norm(ro)


@pytest.mark.parametrize("path", golden_files()[::7], ids=lambda p: p.split("/")[-1][5:-4])
def test_element_kernel_variants_agree(path, tmp_path):
    """The autotuner picks a CTA size per element block; every variant gives
    the same residual (only the order of the FP64 atomic additions differs)."""
    cfg, d = write_golden_case(path, tmp_path)
    m = api.Model.from_json(cfg)
    u = d["u_solve"]
    r_auto = m.residual(u)
    scale = np.linalg.norm(r_auto - m.residual(np.zeros_like(u)))  # |f_int(u)|, the size of what is summed
    info = m.info()
    assert info["elem_threads_fp64"] in (64, 128, 256) and info["elem_threads_fp32"] in (64, 128, 256)
    for t in (64, 128, 256):
        m.set_options(elem_threads=t)
        r = m.residual(u)  # the next device call applies the forced size
        assert m.info()["elem_threads_fp64"] == t
        assert np.linalg.norm(r - r_auto) <= 1e-13 * scale


def test_device_ptrs_refuses_host_memory():
    """With device_ptrs set, pageable host arrays are refused at the ABI
    (cudaPointerGetAttributes) before any kernel could read them."""
    import torch
    m = api.Model.from_case(mg.small_case("C3D8", "nh", "force"))
    m.set_options(device_ptrs=1)
    u_host = np.zeros(m.n_dof)
    with pytest.raises(api.EfemError, match="host memory"):
        m.residual(u_host)
    ut = torch.zeros(m.n_dof, dtype=torch.float64, device="cuda")
    with pytest.raises(api.EfemError, match="host memory"):
        m.residual(ut, np.zeros(m.n_dof))
    with pytest.raises(api.EfemError, match="host memory"):
        m.solve(u_host)
    r = m.residual(ut)  # the model stays usable
    assert torch.isfinite(r).all()
