"""Generate the golden fixtures in this directory from the reference itself.

Run in a container that has the reference tree (the fixtures are committed so
the tests never need it):

    make -C oracle ref
    python tests/golden/make_golden.py            # everything
    python tests/golden/make_golden.py gravity    # the gravity fixtures only
    python tests/golden/make_golden.py trace      # the solve traces only

Each ``case_<etype>_<mat>_<load>.npz`` holds a complete small input (node
coordinates, connectivity, fixed nodes, loads, material) together with what the
reference computes for it through its own public entry points
(oracle/ref_driver.cpp): R(u) at a seeded random u for full and reduced
integration, L(x)I3 applied to a seeded vector (the approximate Jacobian,
src/fe/ElementConstraint.cpp:164-205), and the converged displacement of the
L-BFGS solve with its iteration count.  ``piola_<mat>.npz`` holds P(F) of each
material at seeded random deformation gradients with det F > 0.2.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from efem_b200 import meshgen as mg  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
ETYPES = ["C3D4", "C3D10", "C3D8", "C3D20"]
MATS = ["nh", "mr", "yeoh"]
LOADS = ["pressure", "dpressure", "force"]


def case_arrays(case: mg.Case) -> dict:
    out = {"X": case.mesh.X, "conn": case.mesh.conn.astype(np.int32), "fix": np.asarray(case.fix, dtype=np.int32),
           "materials": json.dumps(case.materials)}
    if case.analysis:
        out["analysis"] = json.dumps(case.analysis)
    for k, (value, faces) in enumerate(case.pressure):
        out[f"pressure{k}_faces"] = np.asarray(faces, dtype=np.int32)
        out[f"pressure{k}_value"] = np.atleast_1d(np.asarray(value, dtype=np.float64))
    for k, (value, nodes) in enumerate(case.force):
        out[f"force{k}_nodes"] = np.asarray(nodes, dtype=np.int32)
        out[f"force{k}_value"] = np.asarray(value, dtype=np.float64)
    return out


def scalar_L_apply(trip, n_dof, v):
    """Apply the reference's 3n x 3n approximate Jacobian to v."""
    out = np.zeros(n_dof)
    np.add.at(out, trip["r"], trip["v"] * v[trip["c"]])
    return out


def gravity_cases():
    """``gravity_<etype>_<consistent|lumped>.npz``: the nodal-force cases with
    analysis.gravity "-z" and a density on the material, the residual at a
    seeded u for both integration rules and the converged solve; the C3D8 pair
    is a dense body under gravity alone (src/fe/InertiaConstraint.cpp:34-84)."""
    rng = np.random.default_rng(20261204)
    for et in ETYPES:
        for consistent in (True, False):
            if et == "C3D8":
                case = mg.small_case(et, "mr", "force")
                case.force = []
                density = 2.0e5
            else:
                case = mg.small_case(et, "nh", "force")
                density = 1100.0
            for m in case.materials:
                m["density"] = density
            case.analysis.update(gravity="-z", consistent_inertia=consistent)
            with tempfile.TemporaryDirectory() as td:
                cfg = case.write(td)
                meta, _ = oracle.run_ref("info", cfg)
                n = meta["n_dof"]
                u = rng.normal(size=n) * 2e-4
                data = case_arrays(case)
                data.update(u=u)
                for integ, red in (("full", False), ("reduced", True)):
                    _, r = oracle.run_ref("residual", cfg, u, reduced=red)
                    data[f"r_{integ}"] = r
                _, r0 = oracle.run_ref("residual", cfg, None)
                meta, us = oracle.run_ref("solve", cfg)
                data.update(r_zero=r0, u_solve=us, solve_meta=json.dumps(meta))
            name = f"gravity_{et}_{'consistent' if consistent else 'lumped'}"
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **data)
            print(name, n, meta["niter"])


TRACE_CASES = [("C3D4", "nh", "force"), ("C3D8", "mr", "pressure"), ("C3D10", "yeoh", "dpressure"),
               ("C3D20", "mr", "pressure"), ("C3D8", "nh", "dpressure"), ("C3D10", "nh", "force")]


def trace_cases():
    """``traces.npz``: the reference's benchmark record (||r||_2 after the
    initial residual and after every line search, LBFGS.h:107-147) of its own
    solve of six small cases, under the key ``<etype>_<mat>_<load>``."""
    out = {}
    for et, mat, load in TRACE_CASES:
        case = mg.small_case(et, mat, load)
        with tempfile.TemporaryDirectory() as td:
            meta, _ = oracle.run_ref("solve", case.write(td), trace=True)
        out[f"{et}_{mat}_{load}"] = meta["trace"]
        print("trace", et, mat, load, meta["niter"], len(meta["trace"]))
    np.savez_compressed(os.path.join(HERE, "traces.npz"), **out)


def main():
    if sys.argv[1:] == ["gravity"]:
        gravity_cases()
        return
    if sys.argv[1:] == ["trace"]:
        trace_cases()
        return
    rng = np.random.default_rng(20261203)
    for et in ETYPES:
        for mat in MATS:
            for load in LOADS:
                case = mg.small_case(et, mat, load)
                with tempfile.TemporaryDirectory() as td:
                    cfg = case.write(td)
                    meta, _ = oracle.run_ref("info", cfg)
                    n = meta["n_dof"]
                    u = rng.normal(size=n) * 2e-4
                    v = rng.normal(size=n)
                    data = case_arrays(case)
                    data.update(u=u, v=v)
                    for integ, red in (("full", False), ("reduced", True)):
                        _, r = oracle.run_ref("residual", cfg, u, reduced=red)
                        _, trip = oracle.run_ref("jacobi", cfg, reduced=red)
                        data[f"r_{integ}"] = r
                        data[f"Kv_{integ}"] = scalar_L_apply(trip, n, v)
                    meta, us = oracle.run_ref("solve", cfg)
                    data["u_solve"] = us
                    data["solve_meta"] = json.dumps(meta)
                    if et == "C3D20":
                        meta, us = oracle.run_ref("solve", cfg, reduced=True)
                        data["u_solve_reduced"] = us
                        data["solve_meta_reduced"] = json.dumps(meta)
                np.savez_compressed(os.path.join(HERE, f"case_{et}_{mat}_{load}.npz"), **data)
                print(et, mat, load, n, meta["niter"])
    # the C3D4 cantilever with follower end pressure (275 nodes, 960 elements)
    case = mg.cantilever_c3d4_pressure()
    with tempfile.TemporaryDirectory() as td:
        cfg = case.write(td)
        meta, us = oracle.run_ref("solve", cfg)
        _, r0 = oracle.run_ref("residual", cfg, None)
        data = case_arrays(case)
        data.update(u_solve=us, solve_meta=json.dumps(meta), r_zero=r0)
        np.savez_compressed(os.path.join(HERE, "cantilever_c3d4_pressure.npz"), **data)
        print("cantilever_c3d4_pressure", meta)
    # material point values
    for mat, (name, C) in {"nh": ("neo_hookean", [114000.0, 0, 0, 0, 1e-6]),
                           "mr": ("mo_riv", [80000.0, 20000.0, 0, 0, 1e-6]),
                           "yeoh": ("yeoh", [110000.0, 0, 20000.0, -300.0, 1e-6])}.items():
        Fs = []
        while len(Fs) < 64:
            F = np.eye(3) + rng.normal(scale=0.25, size=(3, 3))
            if np.linalg.det(F) > 0.2:
                Fs.append(F.T.ravel())  # column-major
        F = np.array(Fs)
        with tempfile.TemporaryDirectory() as td:
            fp, pp = os.path.join(td, "F.f64"), os.path.join(td, "P.f64")
            F.tofile(fp)
            import subprocess
            res = subprocess.run([oracle.REF_BIN, "piola", name] + [repr(c) for c in C] + [fp, pp],
                                 capture_output=True, text=True, check=True)
            P = np.fromfile(pp, dtype=np.float64).reshape(-1, 9)
            kappa = json.loads(res.stdout)["elasticity_coeff"]
        np.savez_compressed(os.path.join(HERE, f"piola_{mat}.npz"), F=F, P=P, C=np.array(C), kappa=kappa)
        print("piola", mat, kappa)
    gravity_cases()
    trace_cases()


if __name__ == "__main__":
    main()
