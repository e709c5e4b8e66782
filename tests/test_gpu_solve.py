"""CUDA L-BFGS solve against the reference's converged displacements."""
import json

import numpy as np
import pytest

import oracle
from conftest import golden_files, write_golden_case
from efem_b200 import api

pytestmark = pytest.mark.gpu
CASES = golden_files()


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.split("/")[-1][5:-4])
def test_solve_identity_h0_matches_oracle(path, tmp_path):
    """nl_solver "lbfgs" (H0 = I/theta): GPU vs the oracle's identical algorithm."""
    cfg, d = write_golden_case(path, tmp_path, nl_solver="lbfgs", max_solver_iters=4000)
    m = api.Model.from_json(cfg)
    u, info = m.solve()
    o = oracle.Oracle(oracle.read_case(cfg))
    uo, io = o.solve()
    assert info["flags"] & api.SOLVE_CONVERGED
    assert info["r_inf"] <= 1e-6
    assert np.linalg.norm(u - uo) <= 1e-6 * np.linalg.norm(uo)
