"""The allocation-free H0 application, efem_precond_apply_noalloc.

Callers that cannot allocate device memory at call time (inside an open CUDA
stream capture, under another framework's caching allocator, or in a loop
that must not synchronise the device) use this entry point instead of
efem_precond_apply.  Its working vectors live in a fixed device array in
place of buffers the model allocates.  Its result must match the regular entry
point's, on consecutive calls that reuse the same array.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden_files, write_golden_case
from efem_b200 import api, meshgen as mg

pytestmark = pytest.mark.gpu


def call_noalloc(model, vt):
    return api.lib().efem_precond_apply_noalloc(model.h, ctypes.c_void_p(vt.data_ptr()))


def build(which, tmp_path):
    if which == "cantilever_c3d4":
        return api.Model.from_case(mg.cantilever_c3d4_pressure())
    path = golden_files("case_C3D20_mr_pressure.npz")[0]
    cfg, _ = write_golden_case(path, tmp_path)
    return api.Model.from_json(cfg)


@pytest.mark.parametrize("which", ["cantilever_c3d4", "c3d20"])
def test_noalloc_matches_precond_apply(which, tmp_path):
    import torch
    m = build(which, tmp_path)
    m.set_options(device_ptrs=1)
    g = torch.Generator(device="cuda").manual_seed(7)
    v = torch.randn(m.n_dof, dtype=torch.float64, device="cuda", generator=g)
    expected = v.clone()
    m.precond_apply(expected)  # the regular entry point (factors on first use)
    torch.cuda.synchronize()
    for _ in range(2):  # two calls in a row share the static array
        out = v.clone()
        assert call_noalloc(m, out) == api.OK, api.last_error()
        torch.cuda.synchronize()
        err = (torch.linalg.norm(out - expected) / torch.linalg.norm(expected)).item()
        assert err <= 1e-12, err


def test_noalloc_needs_a_factor(tmp_path):
    import torch
    m = build("cantilever_c3d4", tmp_path)
    m.set_options(device_ptrs=1)
    m.residual(torch.zeros(m.n_dof, dtype=torch.float64, device="cuda"),
               torch.zeros(m.n_dof, dtype=torch.float64, device="cuda"))
    v = torch.ones(m.n_dof, dtype=torch.float64, device="cuda")
    assert call_noalloc(m, v) == api.ERR_ARG
    assert "factor" in api.last_error()
