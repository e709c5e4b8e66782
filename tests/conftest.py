"""Shared test set-up: the `gpu` marker and golden-fixture helpers."""
import glob
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")

from efem_b200 import meshgen as mg  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_files(pattern="case_*.npz"):
    return sorted(glob.glob(os.path.join(GOLDEN, pattern)))


def case_from_golden(path) -> mg.Case:
    """Rebuild the meshgen.Case stored in a golden fixture."""
    d = np.load(path, allow_pickle=False)
    mesh = mg.Mesh(d["X"], d["conn"].astype(np.int64))
    case = mg.Case(mesh, json.loads(str(d["materials"])), d["fix"])
    if "analysis" in d:
        case.analysis.update(json.loads(str(d["analysis"])))
    k = 0
    while f"pressure{k}_faces" in d:
        v = d[f"pressure{k}_value"]
        value = float(v[0]) if v.shape[0] == 1 else [float(x) for x in v]
        case.pressure.append((value, [tuple(int(x) for x in f) for f in d[f"pressure{k}_faces"]]))
        k += 1
    k = 0
    while f"force{k}_nodes" in d:
        case.force.append(([float(x) for x in d[f"force{k}_value"]], d[f"force{k}_nodes"]))
        k += 1
    return case


def write_golden_case(path, tmpdir, integration="full", **analysis):
    case = case_from_golden(path)
    case.integration = integration
    case.analysis.update(analysis)
    return case.write(str(tmpdir)), np.load(path, allow_pickle=False)


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def write_sample(path, tmpdir):
    """Rebuild the files of a fixture made by make_golden.sample_arrays (a
    config with its mesh and constraint files) under tmpdir, at the relative
    paths the config names; returns (config path, fixture)."""
    d = np.load(path, allow_pickle=False)
    cfg = json.loads(str(d["config"]))
    files = json.loads(str(d["files"]))
    for k, f in enumerate(files):
        out = os.path.join(str(tmpdir), f["path"])
        os.makedirs(os.path.dirname(out), exist_ok=True)
        with open(out, "w") as fh:
            if f["kind"] == "mesh":
                fh.write("#node\n")
                np.savetxt(fh, d[f"file{k}_X"], fmt="%.17g", delimiter="    ")
                fh.write("#element\n")
                tok, ptr = d[f"file{k}_elem"], d[f"file{k}_elem_ptr"]
                for i in range(ptr.shape[0] - 1):
                    fh.write("    ".join(str(int(t)) for t in tok[ptr[i]:ptr[i + 1]]) + "\n")
            else:
                tok, ptr = d[f"file{k}_tok"], d[f"file{k}_ptr"]
                for i in range(ptr.shape[0] - 1):
                    fh.write("    ".join(str(int(t)) for t in tok[ptr[i]:ptr[i + 1]]) + "\n")
    cfg_path = os.path.join(str(tmpdir), "case.json")
    with open(cfg_path, "w") as fh:
        json.dump(cfg, fh, indent=1)
    return cfg_path, d
