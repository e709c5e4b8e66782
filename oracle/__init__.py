"""Test infrastructure: the CPU checkers for the CUDA path.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this package.  It holds

* ``read_case`` -- a Python reader of the reference's input files, following
  src/io/Config.cpp:6-82, src/io/IO.cpp:67-96, src/io/MeshParser.h:22-100,
  src/model/Model.cpp:7-39, src/model/Body.cpp:49-90,
  src/fe/ElementConstraint.cpp:39-67 and src/fe/ExternalConstraint.cpp:13-247;
* ``Oracle`` -- ctypes access to the C restatement in efem_oracle.c;
* ``run_ref`` -- the reference itself, compiled from its own sources into
  _ref/efem_ref by this directory's Makefile.
"""
from __future__ import annotations

import ctypes
import json
import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libefem_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "efem_ref")

MAT_TYPES = {"neo_hookean": 0, "mo_riv": 1, "yeoh": 2}
# analysis.gravity (src/io/Config.cpp:45-62, src/fe/InertiaConstraint.cpp:64-84)
GRAVITY = {"x": (9.8, 0.0, 0.0), "-x": (-9.8, 0.0, 0.0), "y": (0.0, 9.8, 0.0), "-y": (0.0, -9.8, 0.0),
           "z": (0.0, 0.0, 9.8), "-z": (0.0, 0.0, -9.8)}


# --------------------------------------------------------------------------- reader

def _read_lines(path):
    """IO::readFile: trimmed lines, skipping blanks and any line holding '#' or '!'."""
    out = []
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line and "#" not in line and "!" not in line:
                out.append(line)
    return out


def _split(line):
    """boost::split(..., is_any_of(", "), token_compress_on) on a trimmed line."""
    return re.split(r"[, ]+", line)


def read_mesh(path):
    """MeshParser::parse: returns (X (n,3), list of raw element token lists)."""
    nodes, elems = [], []
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    lines = [ln for ln in lines if ln and not ln.startswith("##") and not ln.startswith("!!")]
    i = 0
    while i < len(lines):
        ln = lines[i]
        if ln.startswith("#node"):
            i += 1
            while i < len(lines) and not lines[i].startswith("#"):
                nodes.append([float(t) for t in lines[i].split()[:3]])
                i += 1
            continue
        if ln.startswith("#element"):
            i += 1
            while i < len(lines) and not lines[i].startswith("#"):
                elems.append([int(t) for t in _split(lines[i])])
                i += 1
            continue
        i += 1
    return np.array(nodes, dtype=np.float64).reshape(-1, 3), elems


def _element(tokens):
    """Body::buildElement: node count by token count, optional trailing material id."""
    n = len(tokens)
    nen = 4 if n <= 5 else 8 if n <= 9 else 10 if n <= 11 else 20
    mat = tokens[nen] if n > nen else -1
    return [t - 1 for t in tokens[:nen]], mat


def read_case(cfg_path):
    """Parse a reference config and everything it references into arrays."""
    wd = os.path.dirname(os.path.abspath(cfg_path))
    cfg = json.load(open(cfg_path))
    bodies = []
    for mj in cfg.get("model", []):
        if not isinstance(mj.get("type"), str) or not isinstance(mj.get("mesh_file"), str):
            continue
        if mj.get("pose"):
            raise NotImplementedError("pose transforms are not restated in the oracle")
        X, raw = read_mesh(os.path.join(wd, mj["mesh_file"]))
        bodies.append((mj.get("id", -1), X, raw))
    if len(bodies) != 1:
        raise NotImplementedError("the oracle restates single-body models")
    body_id, X, raw = bodies[0]
    conn, emat = zip(*[_element(t) for t in raw])
    nens = {len(c) for c in conn}
    if len(nens) != 1:
        raise NotImplementedError("the oracle restates single-element-type meshes")
    conn = np.array(conn, dtype=np.int32)
    emat = np.array(emat, dtype=np.int32)
    mats, density = [], []
    for mj in cfg.get("material", []):
        t = mj.get("type")
        if t not in MAT_TYPES:
            continue
        mats.append([MAT_TYPES[t], mj.get("id", -1), mj.get("C10", 0.0), mj.get("C01", 0.0),
                     mj.get("C20", 0.0), mj.get("C30", 0.0), mj.get("D1", 0.0)])
        d = mj.get("density")
        density.append(float(d) if isinstance(d, (int, float)) and not isinstance(d, bool) else 0.0)
    mats = np.array(mats, dtype=np.float64).reshape(-1, 7)
    fixed = np.zeros(X.shape[0], dtype=np.uint8)
    forces, pressures = [], []
    for cj in cfg.get("constraint", []):
        t = cj.get("type")
        fn = cj.get("constraint_file")
        lines = _read_lines(os.path.join(wd, fn)) if isinstance(fn, str) and fn else []
        if t == "fix":
            for ln in lines:
                for tok in _split(ln):
                    fixed[int(tok) - 1] = 1
        elif t == "force":
            nodes = [int(tok) - 1 for ln in lines for tok in _split(ln)]
            forces.append((np.array(cj.get("value", [0, 0, 0]), dtype=np.float64), np.array(nodes, dtype=np.int32)))
        elif t == "pressure":
            faces = []
            for ln in lines:
                face = []
                for tok in _split(ln):
                    v = int(tok) - 1
                    if v not in face:
                        face.append(v)
                faces.append(face)
            pressures.append((cj.get("value"), faces))
    an = cfg.get("analysis", {})
    gravity = an.get("gravity")
    return {
        "X": X, "conn": conn, "elem_mat": emat, "mats": mats, "fixed": fixed,
        "forces": forces, "pressures": pressures,
        "density": np.array(density, dtype=np.float64),
        "gravity": GRAVITY.get(gravity) if isinstance(gravity, str) else None,
        "consistent_inertia": an.get("consistent_inertia") is True,
        "reduced": an.get("integration", "full") == "reduced",
        "epsilon": float(an.get("residual_criterion", 1e-6)),
        "max_iterations": int(an.get("max_solver_iters", 0)),
        "max_linesearch": int(an.get("max_line_search", 20)),
        "use_precond": an.get("nl_solver", "lbfgs_ah") != "lbfgs",
    }


# --------------------------------------------------------------------------- C restatement

class _Params(ctypes.Structure):
    _fields_ = [("epsilon", ctypes.c_double), ("max_iterations", ctypes.c_int),
                ("max_linesearch", ctypes.c_int), ("m", ctypes.c_int), ("use_precond", ctypes.c_int)]


class _Info(ctypes.Structure):
    _fields_ = [("niter", ctypes.c_int), ("r_evals", ctypes.c_int), ("precond_ok", ctypes.c_int),
                ("u_inf", ctypes.c_double), ("r_inf", ctypes.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
        L = ctypes.CDLL(LIB_PATH)
        dp, ip = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, dp, ctypes.c_int, ctypes.c_int, ip, ip, ctypes.c_int, dp,
                                 ctypes.POINTER(ctypes.c_ubyte), ctypes.c_int]
        L.orc_add_pressure.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ip, ctypes.c_double, dp]
        L.orc_add_force.argtypes = [ctypes.c_void_p, ctypes.c_int, ip, dp]
        L.orc_add_gravity.argtypes = [ctypes.c_void_p, dp, ctypes.c_int, dp]
        L.orc_set_trace.argtypes = [ctypes.c_void_p, dp, ctypes.c_int]
        L.orc_trace_count.argtypes = [ctypes.c_void_p]
        L.orc_n_dof.argtypes = [ctypes.c_void_p]
        L.orc_n_elem_skipped.argtypes = [ctypes.c_void_p]
        L.orc_residual.argtypes = [ctypes.c_void_p, dp, dp]
        L.orc_approx_jacobian_dense.argtypes = [ctypes.c_void_p, dp]
        L.orc_solve.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Params), dp, ctypes.POINTER(_Info)]
        L.orc_precond_apply.argtypes = [ctypes.c_void_p, dp]
        L.orc_piola.argtypes = [ctypes.c_int, dp, ctypes.c_int, dp, dp]
        L.orc_elasticity_coeff.restype = ctypes.c_double
        L.orc_elasticity_coeff.argtypes = [ctypes.c_int, dp]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


class Oracle:
    """The C restatement built from a ``read_case`` dictionary."""

    def __init__(self, case):
        L = lib()
        self.case = case
        X = np.ascontiguousarray(case["X"], dtype=np.float64)
        conn = np.ascontiguousarray(case["conn"], dtype=np.int32)
        emat = np.ascontiguousarray(case["elem_mat"], dtype=np.int32)
        mats = np.ascontiguousarray(case["mats"], dtype=np.float64)
        fixed = np.ascontiguousarray(case["fixed"], dtype=np.uint8)
        self.h = L.orc_create(X.shape[0], _p(X), conn.shape[0], conn.shape[1], _p(conn, ctypes.c_int),
                              _p(emat, ctypes.c_int), mats.shape[0], _p(mats), _p(fixed, ctypes.c_ubyte),
                              int(case["reduced"]))
        if not self.h:
            raise ValueError("oracle: unsupported element type")
        for value, nodes in case["forces"]:
            v = np.ascontiguousarray(value, dtype=np.float64)
            nd = np.ascontiguousarray(nodes, dtype=np.int32)
            L.orc_add_force(self.h, nd.shape[0], _p(nd, ctypes.c_int), _p(v))
        for value, faces in case["pressures"]:
            by_nn = {}
            for f in faces:
                by_nn.setdefault(len(f), []).append(f)
            for nn, fs in by_nn.items():
                arr = np.ascontiguousarray(fs, dtype=np.int32)
                if isinstance(value, (list, tuple)):
                    dv = np.ascontiguousarray(value, dtype=np.float64)
                    rc = L.orc_add_pressure(self.h, arr.shape[0], nn, _p(arr, ctypes.c_int), 0.0, _p(dv))
                else:
                    rc = L.orc_add_pressure(self.h, arr.shape[0], nn, _p(arr, ctypes.c_int), float(value or 0.0), None)
                if rc != 0:
                    raise ValueError(f"oracle: pressure face setup failed ({rc})")
        if case.get("gravity") is not None:
            g = np.ascontiguousarray(case["gravity"], dtype=np.float64)
            rho = np.ascontiguousarray(case["density"], dtype=np.float64)
            if rho.size == 0:
                rho = np.zeros(1)
            L.orc_add_gravity(self.h, _p(g), int(case["consistent_inertia"]), _p(rho))
        self.n_dof = L.orc_n_dof(self.h)

    def residual(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        r = np.zeros(self.n_dof)
        lib().orc_residual(self.h, _p(u), _p(r))
        return r

    def approx_jacobian_dense(self):
        n = self.n_dof // 3
        L = np.zeros((n, n))
        lib().orc_approx_jacobian_dense(self.h, _p(L))
        return L

    def solve(self, u0=None, trace=0, **over):
        """L-BFGS solve; with trace > 0 the info dict also holds "trace", an
        (records, 5) array (0, ||r||_2, ||r||_inf, step, residual evaluations)."""
        c = dict(self.case)
        c.update(over)
        p = _Params(c["epsilon"], c["max_iterations"], c["max_linesearch"], c.get("m", 6), int(c["use_precond"]))
        u = np.zeros(self.n_dof) if u0 is None else np.array(u0, dtype=np.float64)
        info = _Info()
        buf = np.zeros((max(trace, 1), 5))
        lib().orc_set_trace(self.h, _p(buf) if trace > 0 else None, int(trace))
        lib().orc_solve(self.h, ctypes.byref(p), _p(u), ctypes.byref(info))
        out = {"niter": info.niter, "r_evals": info.r_evals, "precond_ok": info.precond_ok,
               "u_inf": info.u_inf, "r_inf": info.r_inf}
        if trace > 0:
            out["trace"] = buf[:min(trace, lib().orc_trace_count(self.h))].copy()
        lib().orc_set_trace(self.h, None, 0)
        return u, out

    def precond_apply(self, v):
        """H0 v with H0 the inverse approximate Jacobian; None if L is not SPD."""
        v = np.array(v, dtype=np.float64)
        ok = lib().orc_precond_apply(self.h, _p(v))
        return v if ok else None

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None


def piola(mat_type, C, F):
    """P(F) for column-major F of shape (n, 9)."""
    F = np.ascontiguousarray(F, dtype=np.float64)
    C = np.ascontiguousarray(C, dtype=np.float64)
    P = np.zeros_like(F)
    lib().orc_piola(int(mat_type), _p(C), F.shape[0], _p(F), _p(P))
    return P


# --------------------------------------------------------------------------- the reference

def ref_available():
    return os.path.exists(REF_BIN)


def run_ref(cmd, cfg, *args, reduced=False, trace=False, timeout=3600):
    """Run the reference driver; returns (parsed JSON line, output arrays).
    ``trace`` (solve only) adds meta["trace"]: the reference's benchmark
    record of ||r||_2, initial residual first, then one per line search."""
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "out.bin")
        tpath = os.path.join(td, "trace.f64")
        argv = [REF_BIN, cmd, cfg]
        if cmd == "residual":
            u = args[0]
            if u is None:
                argv.append("zero")
            else:
                up = os.path.join(td, "u.f64")
                np.ascontiguousarray(u, dtype=np.float64).tofile(up)
                argv.append(up)
        argv.append(out)
        if reduced:
            argv.append("--reduced")
        argv += [str(a) for a in args[1:]] if cmd == "residual" else [str(a) for a in args]
        if trace:
            argv += ["--trace", tpath]
        res = subprocess.run(argv, capture_output=True, text=True, timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError(f"efem_ref {cmd} failed: {res.stderr[-500:]}")
        meta = json.loads(res.stdout.strip().splitlines()[-1])
        if trace:
            meta["trace"] = np.fromfile(tpath, dtype=np.float64)
        if cmd == "jacobi":
            raw = open(out, "rb").read()
            cnt = np.frombuffer(raw[:8], dtype=np.int64)[0]
            rec = np.frombuffer(raw[8:], dtype=np.dtype([("r", "<i4"), ("c", "<i4"), ("v", "<f8")]), count=cnt)
            return meta, rec
        if cmd == "info":
            return meta, np.fromfile(out, dtype=np.int32)
        return meta, np.fromfile(out, dtype=np.float64)
