"""Generate the golden fixtures in this directory from the reference itself.

Run in a container that has the reference tree (the fixtures are committed so
the tests never need it):

    make -C oracle ref
    python tests/golden/make_golden.py            # everything
    python tests/golden/make_golden.py gravity    # the gravity fixtures only
    python tests/golden/make_golden.py trace      # the solve traces only
    python tests/golden/make_golden.py samples    # the reference's own sample problems
    python tests/golden/make_golden.py configs    # converged u of the large benchmark meshes
    python tests/golden/make_golden.py multibody  # two bodies with pose and model_id routing
    python tests/golden/make_golden.py failure    # a singular approximate Jacobian (fallback solve)
    python tests/golden/make_golden.py batch      # three members of the benchmark batch

``samples`` and ``configs`` read the reference tree: its location is the
EFEM_REFERENCE environment variable, else a ``reference`` directory beside
this repository.

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


def reference_root():
    """The reference tree: $EFEM_REFERENCE, else ``reference`` beside this repository."""
    return os.environ.get("EFEM_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")


# The reference's own sample problems (sample/<problem>/<problem>.json); each
# config names one element variant's files, the others are selected by
# switching the variant directory in every path (as its README describes).
REF_SAMPLES = [("beam", "c3d4"), ("beam", "c3d20"), ("cap", "c3d4"), ("cap", "c3d20"),
               ("finger", "c3d4"), ("finger", "c3d10")]


def _ragged(rows):
    flat = np.array([t for r in rows for t in r], dtype=np.int32)
    ptr = np.cumsum([0] + [len(r) for r in rows]).astype(np.int64)
    return flat, ptr


def _int_lines(path):
    """Integer token lists of a constraint file's lines (src/io/IO.cpp:67-96)."""
    return [[int(t) for t in oracle._split(ln)] for ln in oracle._read_lines(path)]


def sample_arrays(cfg_path):
    """Everything a sample's config reads, as arrays: node coordinates and
    element token lists of each mesh file, integer token lines of each
    constraint file, and the config text itself."""
    wd = os.path.dirname(os.path.abspath(cfg_path))
    cfg = json.load(open(cfg_path))
    out = {"config": json.dumps(cfg)}
    files = []
    for mj in cfg["model"]:
        X, raw = oracle.read_mesh(os.path.join(wd, mj["mesh_file"]))
        k = len(files)
        files.append({"path": mj["mesh_file"], "kind": "mesh"})
        out[f"file{k}_X"] = X
        out[f"file{k}_elem"], out[f"file{k}_elem_ptr"] = _ragged(raw)
    for cj in cfg["constraint"]:
        fn = cj.get("constraint_file")
        if not isinstance(fn, str) or not fn:
            continue
        k = len(files)
        files.append({"path": fn, "kind": "lines"})
        out[f"file{k}_tok"], out[f"file{k}_ptr"] = _ragged(_int_lines(os.path.join(wd, fn)))
    out["files"] = json.dumps(files)
    return out


def reference_samples():
    """``sample_<problem>_<variant>.npz``: the reference's six sample problems
    (its own meshes, loads and materials, read in place) with the reference's
    converged displacement at the config's own tolerance (``u_solve``) and at
    a residual of 1e-10 N (``u_tight``)."""
    import shutil
    src = os.path.join(reference_root(), "sample")
    for prob, var in REF_SAMPLES:
        cfg = json.load(open(os.path.join(src, prob, f"{prob}.json")))
        base_var = cfg["model"][0]["mesh_file"].split("/")[0]
        swap = lambda p: var + p[len(base_var):] if p.startswith(base_var + "/") else p
        for mj in cfg["model"]:
            mj["mesh_file"] = swap(mj["mesh_file"])
        for cj in cfg["constraint"]:
            if isinstance(cj.get("constraint_file"), str):
                cj["constraint_file"] = swap(cj["constraint_file"])
        with tempfile.TemporaryDirectory() as td:
            os.makedirs(os.path.join(td, var))
            for fn in os.listdir(os.path.join(src, prob, var)):
                shutil.copy(os.path.join(src, prob, var, fn), os.path.join(td, var, fn))
            path = os.path.join(td, f"{prob}.json")
            json.dump(cfg, open(path, "w"), indent=1)
            data = sample_arrays(path)
            meta, us = oracle.run_ref("solve", path)
            data.update(u_solve=us, solve_meta=json.dumps(meta))
            cfg["analysis"]["residual_criterion"] = 1e-10
            json.dump(cfg, open(path, "w"), indent=1)
            meta_t, ut = oracle.run_ref("solve", path)
            data.update(u_tight=ut, solve_meta_tight=json.dumps(meta_t))
        np.savez_compressed(os.path.join(HERE, f"sample_{prob}_{var}.npz"), **data)
        print("sample", prob, var, meta["niter"], meta_t["niter"], meta["solve_s"], meta_t["solve_s"])


def config_case(name):
    """The large benchmark meshes by name: (case, reduced)."""
    if name == "beam_c3d8_mr_force":
        return mg.cantilever_c3d8_force(), False
    if name == "cap_c3d20r_nh_pressure":
        return mg.cylinder_cap_c3d20(), True
    if name == "finger_c3d10_yeoh_pressure":
        return mg.finger_c3d10()[0], False
    raise ValueError(name)


CONFIG_CASES = ["beam_c3d8_mr_force", "cap_c3d20r_nh_pressure", "finger_c3d10_yeoh_pressure"]


def mesh_digest(case):
    """A short fingerprint of a generated mesh (coordinates, connectivity, fixed nodes)."""
    import hashlib
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(case.mesh.X, dtype=np.float64).tobytes())
    h.update(np.ascontiguousarray(case.mesh.conn, dtype=np.int64).tobytes())
    h.update(np.ascontiguousarray(case.fix, dtype=np.int64).tobytes())
    return h.hexdigest()[:16]


def config_cases(names=None, eps=1e-6):
    """``config_<name>.npz``: the reference's converged displacement (stored
    as float32, ample for the 1e-6 and 1e-4 relative comparisons) of the
    generated benchmark meshes -- the C3D8 Mooney-Rivlin beam under tip
    forces, the C3D20R cylinder cap under 10 kPa and the C3D10 Yeoh finger
    under 30 kPa -- with the generator's mesh fingerprint.  The meshes are
    regenerated by the tests from efem_b200.meshgen."""
    for name in names or CONFIG_CASES:
        case, red = config_case(name)
        case.analysis["residual_criterion"] = eps
        with tempfile.TemporaryDirectory() as td:
            cfg = case.write(td)
            meta, us = oracle.run_ref("solve", cfg, reduced=red, timeout=48 * 3600)
        save_config_fixture(name, case, meta, us, eps)


def save_config_fixture(name, case, meta, us, eps):
    np.savez_compressed(os.path.join(HERE, f"config_{name}.npz"), u_solve=us.astype(np.float32),
                        u_norm=np.linalg.norm(us), solve_meta=json.dumps(meta), mesh=mesh_digest(case),
                        epsilon=eps)
    print("config", name, meta)


def multibody_case(td):
    """Two bodies built from one C3D10 mesh with trailing per-element material
    ids, placed by ``pose`` (body 1: translation; body 2: Euler angles, scale,
    axis-angle rotation and translation), with constraints routed by
    ``model_id``: both bodies fixed at their x = 0 face, a follower pressure on
    body 2's end face, a nodal force on body 1's end nodes
    (src/model/Model.cpp:14-37, src/math/Math.cpp:37-99,
    src/fe/ExternalConstraint.cpp:65-81)."""
    base = mg.small_case("C3D10", "nh", "pressure", seed=3)
    m = base.mesh
    ne = m.conn.shape[0]
    m.mat = np.where(np.arange(ne) % 3 == 0, 2, 1).astype(np.int64)
    mg.write_mesh(os.path.join(td, "mesh.txt"), m)
    mg.write_nodes(os.path.join(td, "fix.txt"), base.fix)
    mg.write_faces(os.path.join(td, "pressure.txt"), base.pressure[0][1])
    tip = mg.nodes_where(m, lambda X: np.abs(X[:, 0] - 0.03) < 1e-9)
    mg.write_nodes(os.path.join(td, "force.txt"), tip)
    cfg = {
        "analysis": {"max_solver_iters": 0, "max_line_search": 20, "residual_criterion": 1e-8},
        "model": [
            {"id": 1, "type": "soft", "mesh_file": "mesh.txt", "pose": [{"t": [0.0, 0.05, 0.0]}]},
            {"id": 2, "type": "soft", "mesh_file": "mesh.txt",
             "pose": [{"r": [10.0, -20.0, 30.0]}, {"s": [1.2, 0.9, 1.1]}, {"r": [1.0, 2.0, 2.0, 45.0]},
                      {"t": [0.01, -0.02, 0.03]}]},
        ],
        "constraint": [
            {"id": 1, "type": "fix", "constraint_file": "fix.txt", "model_id": [1, 2]},
            {"id": 2, "type": "pressure", "value": 2.0e4, "constraint_file": "pressure.txt", "model_id": 2},
            {"id": 3, "type": "force", "value": [0.0, 0.0, -0.05], "constraint_file": "force.txt", "model_id": [1]},
        ],
        "material": [
            {"id": 1, "type": "neo_hookean", "C10": 114000.0, "D1": 1e-6, "density": 1050.0},
            {"id": 2, "type": "yeoh", "C10": 110000.0, "C20": 20000.0, "C30": -300.0, "D1": 1e-6,
             "density": 1050.0},
        ],
        "output": {"save_frame": False, "show_log": False, "disk_log": False},
    }
    path = os.path.join(td, "multibody.json")
    json.dump(cfg, open(path, "w"), indent=1)
    return path


def multibody():
    """``multibody_c3d10_pose.npz``: the two-body case's inputs, the
    reference's R(u) at a seeded u and its converged displacement."""
    rng = np.random.default_rng(20261205)
    with tempfile.TemporaryDirectory() as td:
        cfg = multibody_case(td)
        data = sample_arrays(cfg)
        meta, _ = oracle.run_ref("info", cfg)
        u = rng.normal(size=meta["n_dof"]) * 2e-4
        _, r = oracle.run_ref("residual", cfg, u)
        meta, us = oracle.run_ref("solve", cfg)
        data.update(u=u, r=r, u_solve=us, solve_meta=json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "multibody_c3d10_pose.npz"), **data)
    print("multibody", meta)


def failure_cases():
    """``failure_orphan_node.npz``: the C3D10 Neo-Hookean pressure case with
    one more node that no element uses.  The node is free, so the scalar
    approximate Jacobian has a zero row and the reference's factorisation
    fails; its solve falls back to H0 = I/theta (src/simulation/nlsolver/
    LBFGS.h:65-81).  Holds the reference's solution at 1e-6 N (``u_solve``)
    and at 1e-10 N (``u_tight``) and the orphan node's first DOF."""
    case = mg.small_case("C3D10", "nh", "pressure")
    X = case.mesh.X
    case.mesh = mg.Mesh(np.vstack([X, [[0.05, 0.02, 0.02]]]), case.mesh.conn, case.mesh.mat)
    data = case_arrays(case)
    with tempfile.TemporaryDirectory() as td:
        cfg = case.write(td)
        meta, us = oracle.run_ref("solve", cfg)
        assert meta["precond_ok"] == 0, meta
        case.analysis.update(residual_criterion=1e-10)
        cfg = case.write(td)
        meta_t, ut = oracle.run_ref("solve", cfg)
    n_free = X.shape[0] + 1 - len(case.fix)
    data.update(u_solve=us, solve_meta=json.dumps(meta), u_tight=ut, solve_meta_tight=json.dumps(meta_t),
                orphan_dof=3 * (n_free - 1))
    np.savez_compressed(os.path.join(HERE, "failure_orphan_node.npz"), **data)
    print("failure_orphan_node", meta, meta_t["niter"])


BATCH_SEED = 20261203


def batch_members():
    """``batch_member_<k>.npz``: three members of the benchmark batch
    (efem_b200.meshgen.batch_beams(seed=20261203), the three with the fewest
    elements), the reference's solution of each at 1e-6 N (``u_solve``) and at
    1e-10 N (``u_tight``), with the member's index in the batch."""
    cases = mg.batch_beams(seed=BATCH_SEED)
    order = sorted(range(len(cases)), key=lambda i: cases[i].mesh.conn.shape[0])[:3]
    for k, i in enumerate(order):
        case = cases[i]
        data = case_arrays(case)
        with tempfile.TemporaryDirectory() as td:
            cfg = case.write(td)
            meta, us = oracle.run_ref("solve", cfg)
            case.analysis.update(residual_criterion=1e-10)
            cfg = case.write(td)
            meta_t, ut = oracle.run_ref("solve", cfg)
        data.update(u_solve=us, solve_meta=json.dumps(meta), u_tight=ut, solve_meta_tight=json.dumps(meta_t),
                    member=i)
        np.savez_compressed(os.path.join(HERE, f"batch_member_{k}.npz"), **data)
        print("batch member", i, case.mesh.conn.shape[0], meta["niter"], meta_t["niter"])


def inverted_cases():
    """``inverted_<et>_<mat>.npz``: the reference's residual at a displacement
    that turns every element inside out (x -> -X/2 along the beam axis plus a
    seeded perturbation, so J is about -1/2 at every Gauss point).  The
    reference's laws take J^{-2/3} as (J^2)^{-1/3} and stay finite there; a
    solve whose line search tries such a state (the C3D8 beam under tip forces
    does at its seventh iteration) takes its next step from these values."""
    rng = np.random.default_rng(20261204)
    for et in ("C3D4", "C3D8", "C3D10", "C3D20"):
        for mat in MATS:
            case = mg.small_case(et, mat, "force")
            with tempfile.TemporaryDirectory() as td:
                cfg = case.write(td)
                meta, _ = oracle.run_ref("info", cfg)
                n = meta["n_dof"]
                # free nodes in the reference's DOF order: the fixture stores u per DOF
                _, r0 = oracle.run_ref("residual", cfg, None)
                free = np.setdiff1d(np.arange(case.mesh.X.shape[0]), np.asarray(case.fix))
                X = case.mesh.X[free]
                assert 3 * X.shape[0] == n
                h = np.ptp(case.mesh.X[:, 0]) / 10.0
                u = np.zeros((X.shape[0], 3))
                u[:, 0] = -1.5 * X[:, 0]
                u += rng.normal(scale=0.02 * h, size=u.shape)
                u = u.ravel()
                data = case_arrays(case)
                data.update(u=u)
                _, r = oracle.run_ref("residual", cfg, u)
                data["r_full"] = r
                if et == "C3D20":
                    _, rr = oracle.run_ref("residual", cfg, u, reduced=True)
                    data["r_reduced"] = rr
            assert np.all(np.isfinite(data["r_full"]))
            np.savez_compressed(os.path.join(HERE, f"inverted_{et}_{mat}.npz"), **data)
            print("inverted", et, mat, n, float(np.abs(data["r_full"]).max()))


def beam_record(iters=12):
    """``config_beam_c3d8_mr_force_record.npz``: the reference's own solve of
    the C3D8 Mooney-Rivlin beam under 0.5 N tip forces does not converge: at
    its seventh iteration the line search accepts a state with elements
    turned inside out and ||r|| grows without bound (1e93 N by iteration 30).
    Its converged displacement therefore does not exist; what pins this
    configuration is its benchmark record (||r||_2 after every line search,
    initial residual first) over the first iterations, and the steps and
    residual evaluations of the same solve from the C restatement (oracle),
    which follows the same record."""
    case, _ = config_case("beam_c3d8_mr_force")
    with tempfile.TemporaryDirectory() as td:
        cfg = case.write(td)
        meta, _ = oracle.run_ref("solve", cfg, "--max-iters", str(iters), trace=True, timeout=3600)
        o = oracle.Oracle(oracle.read_case(cfg))
    _, info = o.solve(max_iterations=iters, trace=iters + 1)
    rec = np.asarray(meta.pop("trace"))
    np.savez_compressed(os.path.join(HERE, "config_beam_c3d8_mr_force_record.npz"), r_norm2=rec,
                        oracle_trace=info["trace"], solve_meta=json.dumps(meta), mesh=mesh_digest(case))
    print("beam record", meta, rec[:iters + 1])


def main():
    if sys.argv[1:] == ["beamrecord"]:
        beam_record()
        return
    if sys.argv[1:] == ["inverted"]:
        inverted_cases()
        return
    if sys.argv[1:] == ["gravity"]:
        gravity_cases()
        return
    if sys.argv[1:] == ["trace"]:
        trace_cases()
        return
    if sys.argv[1:2] == ["samples"]:
        reference_samples()
        return
    if sys.argv[1:2] == ["configs"]:
        config_cases(sys.argv[2:] or None)
        return
    if sys.argv[1:] == ["multibody"]:
        multibody()
        return
    if sys.argv[1:] == ["failure"]:
        failure_cases()
        return
    if sys.argv[1:] == ["batch"]:
        batch_members()
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
