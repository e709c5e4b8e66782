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


def test_noalloc_inside_a_graph_capture(tmp_path):
    """The use the entry point exists for: recorded into a CUDA graph on the
    caller's stream (efem_set_stream names the capturing stream), then
    replayed; each replay gives the regular entry point's result."""
    import torch
    m = build("cantilever_c3d4", tmp_path)
    m.set_options(device_ptrs=1)
    g = torch.Generator(device="cuda").manual_seed(11)
    v = torch.randn(m.n_dof, dtype=torch.float64, device="cuda", generator=g)
    expected = v.clone()
    m.precond_apply(expected)
    buf = v.clone()
    assert call_noalloc(m, buf) == api.OK, api.last_error()  # first call on the device: outside any capture
    s = torch.cuda.Stream()
    m.set_stream(s.cuda_stream)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        buf.copy_(v)
        torch.cuda.synchronize()
        with torch.cuda.graph(graph, stream=s):
            assert call_noalloc(m, buf) == api.OK, api.last_error()
    for _ in range(2):
        buf.copy_(v)
        graph.replay()
        torch.cuda.synchronize()
        err = (torch.linalg.norm(buf - expected) / torch.linalg.norm(expected)).item()
        assert err <= 1e-12, err
    m.set_stream(None)
    del graph


def test_noalloc_refuses_a_model_beyond_the_workspace():
    """A model whose two work vectors alone exceed the static array (more
    than 349 525 free nodes) is refused with EFEM_ERR_ARG and the sizes in
    the message, before any device work."""
    import torch
    n = 350_000
    X = np.zeros((n, 3))
    X[:4] = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]
    X[4:, 0] = 2.0 + np.arange(n - 4) * 1e-3
    m = api.Model.from_arrays(X, [(np.array([[0, 1, 2, 3]]), None)], [{"type": "neo_hookean", "C10": 1e5, "D1": 1e-6}],
                              [("fix", np.array([0]))])
    v = torch.zeros(8, dtype=torch.float64, device="cuda")
    assert call_noalloc(m, v) == api.ERR_ARG
    msg = api.last_error()
    assert "workspace" in msg and str(2 << 20) in msg, msg
