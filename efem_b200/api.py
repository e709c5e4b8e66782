"""Python access to libefem_b200.so (the C ABI declared in include/efem_gpu.h).

The library is the product: C++ host set-up and hand-written sm_100a CUDA
kernels.  This module only marshals arguments.  It never computes a result
itself, and it raises when the library or a GPU is missing.

``Simulator`` mirrors the reference's JSON-driven entry point
(``Simulator::initial(path)`` / ``Simulator::start()``,
src/simulation/Simulator.cpp:6-41).  ``Model`` exposes the hot-path calls one
by one: ``residual`` (``SoftObjective::residual``), ``solve``
(``LBFGSSolver::solve``), ``approx_jacobian_csr`` (``Constraint::getJacobi``)
and ``precond_apply`` (the ``SimplicialLLT::solve`` of ``LBFGSMat::apply_Hv``).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libefem_b200.so")

OK, ERR_ARG, ERR_CONFIG, ERR_MESH, ERR_CUDA, ERR_NAN, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_NO_DEVICE, ERR_FACE = range(10)
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_CONFIG", 3: "ERR_MESH", 4: "ERR_CUDA", 5: "ERR_NAN",
                6: "ERR_TIMEOUT", 7: "ERR_UNSUPPORTED", 8: "ERR_NO_DEVICE", 9: "ERR_FACE"}
NEO_HOOKEAN, MOONEY_RIVLIN, YEOH = 0, 1, 2
LOAD_FIX, LOAD_FORCE, LOAD_PRESSURE, LOAD_DPRESSURE, LOAD_GRAVITY = 0, 1, 2, 3, 4
# analysis "gravity" strings (src/io/Config.cpp:45-62) as accelerations
GRAVITY = {"x": (9.8, 0.0, 0.0), "-x": (-9.8, 0.0, 0.0), "y": (0.0, 9.8, 0.0), "-y": (0.0, -9.8, 0.0),
           "z": (0.0, 0.0, 9.8), "-z": (0.0, 0.0, -9.8)}
FP64, MIXED = 0, 1
SOLVE_CONVERGED, SOLVE_PRECOND_FALLBACK, SOLVE_DX_CONVERGED, SOLVE_MAX_ITERS, SOLVE_PDL, SOLVE_REFINED = 1, 2, 4, 8, 16, 32
SOLVE_BATCHED = 64

EXPORTED = ["efem_default_options", "efem_model_create_from_json", "efem_model_create", "efem_model_destroy",
            "efem_get_options", "efem_set_options", "efem_get_model_info", "efem_dof_map", "efem_residual",
            "efem_approx_jacobian_csr", "efem_precond_apply", "efem_precond_apply_noalloc", "efem_solve",
            "efem_set_stream", "efem_last_error", "efem_version", "efem_hvp", "efem_hvp_transpose",
            "efem_residual_param_derivative", "efem_adjoint", "efem_strain_energy", "efem_write_vtk",
            "efem_batch_solve", "efem_external_load", "efem_solve_trace", "efem_fma_peak"]


class EfemError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("integration", ctypes.c_int), ("nl_solver", ctypes.c_int),
                ("m", ctypes.c_int), ("max_iterations", ctypes.c_int), ("max_linesearch", ctypes.c_int),
                ("residual_criterion", ctypes.c_double), ("dx_criterion", ctypes.c_double),
                ("device_ptrs", ctypes.c_int), ("deterministic", ctypes.c_int), ("device", ctypes.c_int),
                ("host_loop", ctypes.c_int), ("adjoint_tolerance", ctypes.c_double),
                ("adjoint_max_iterations", ctypes.c_int), ("elem_threads", ctypes.c_int),
                ("consistent_inertia", ctypes.c_int), ("trace", ctypes.c_int),
                ("solve_subtree_levels", ctypes.c_int), ("line_search", ctypes.c_int),
                ("wait_limit", ctypes.c_int), ("wait_test", ctypes.c_int)]


class SolveInfo(ctypes.Structure):
    _fields_ = [("niter", ctypes.c_int), ("n_residual_evals", ctypes.c_int), ("n_jacobian_evals", ctypes.c_int),
                ("flags", ctypes.c_int), ("u_inf", ctypes.c_double), ("r_inf", ctypes.c_double),
                ("ms_total", ctypes.c_double), ("ms_factor", ctypes.c_double), ("ms_residual", ctypes.c_double),
                ("ms_precond", ctypes.c_double), ("n_kernel_launches", ctypes.c_longlong),
                ("n_precond_applies", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AdjointInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("flags", ctypes.c_int), ("rel_residual", ctypes.c_double),
                ("ms_total", ctypes.c_double), ("ms_solve", ctypes.c_double), ("ms_params", ctypes.c_double),
                ("n_kernel_launches", ctypes.c_longlong), ("solve_bytes", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ModelInfo(ctypes.Structure):
    _fields_ = [("n_nodes", ctypes.c_int), ("n_free_nodes", ctypes.c_int), ("n_dof", ctypes.c_int),
                ("n_elements", ctypes.c_int), ("n_elements_skipped", ctypes.c_int), ("n_faces", ctypes.c_int),
                ("n_force_nodes", ctypes.c_int), ("n_blocks", ctypes.c_int), ("factor_nnz", ctypes.c_longlong),
                ("n_supernodes", ctypes.c_int), ("n_levels", ctypes.c_int), ("factor_gflop", ctypes.c_double),
                ("factor_dinv_nnz", ctypes.c_longlong), ("residual_bytes", ctypes.c_longlong),
                ("residual_flops", ctypes.c_double), ("n_params", ctypes.c_int),
                ("elem_threads_fp64", ctypes.c_int), ("elem_threads_fp32", ctypes.c_int),
                ("solve_subtree_levels", ctypes.c_int), ("n_solve_subtrees", ctypes.c_int),
                ("solve_ctas", ctypes.c_int), ("solve_smem_bytes", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Material(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("id", ctypes.c_int), ("C10", ctypes.c_double), ("C01", ctypes.c_double),
                ("C20", ctypes.c_double), ("C30", ctypes.c_double), ("D1", ctypes.c_double),
                ("density", ctypes.c_double)]


class ElementBlock(ctypes.Structure):
    _fields_ = [("nen", ctypes.c_int), ("n_elem", ctypes.c_int), ("conn", ctypes.POINTER(ctypes.c_int)),
                ("material_id", ctypes.POINTER(ctypes.c_int))]


class MeshDesc(ctypes.Structure):
    _fields_ = [("n_nodes", ctypes.c_int), ("X", ctypes.POINTER(ctypes.c_double)), ("n_blocks", ctypes.c_int),
                ("blocks", ctypes.POINTER(ElementBlock))]


class LoadDesc(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("n", ctypes.c_int), ("nodes", ctypes.POINTER(ctypes.c_int)),
                ("face_ptr", ctypes.POINTER(ctypes.c_int)), ("value", ctypes.c_double * 3)]


_lib = None


def lib():
    """Load libefem_b200.so (built by ``__graft_entry__.build()``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EfemError(ERR_UNSUPPORTED, f"{LIB_PATH} is not built; run __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        sig = {
            "efem_default_options": [ctypes.POINTER(Options)],
            "efem_model_create_from_json": [ctypes.c_char_p, ctypes.POINTER(vp)],
            "efem_model_create": [ctypes.POINTER(MeshDesc), ctypes.POINTER(Material), ctypes.c_int,
                                  ctypes.POINTER(LoadDesc), ctypes.c_int, ctypes.POINTER(Options), ctypes.POINTER(vp)],
            "efem_model_destroy": [vp],
            "efem_get_options": [vp, ctypes.POINTER(Options)],
            "efem_set_options": [vp, ctypes.POINTER(Options)],
            "efem_get_model_info": [vp, ctypes.POINTER(ModelInfo)],
            "efem_dof_map": [vp, ip],
            "efem_residual": [vp, vp, vp],
            "efem_approx_jacobian_csr": [vp, ctypes.POINTER(ctypes.c_longlong), ip, ip, dp],
            "efem_precond_apply": [vp, vp],
            "efem_solve": [vp, vp, ctypes.POINTER(SolveInfo)],
            "efem_last_error": [ctypes.c_char_p, ctypes.c_size_t],
            "efem_set_stream": [vp, vp],
            "efem_precond_apply_noalloc": [vp, vp],
            "efem_hvp": [vp, vp, vp, vp],
            "efem_hvp_transpose": [vp, vp, vp, vp],
            "efem_residual_param_derivative": [vp, vp, ctypes.c_int, vp],
            "efem_adjoint": [vp, vp, vp, dp, vp, ctypes.POINTER(AdjointInfo)],
            "efem_strain_energy": [vp, vp, dp],
            "efem_write_vtk": [vp, vp, ctypes.c_char_p],
            "efem_batch_solve": [ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(SolveInfo),
                                 ctypes.c_int],
            "efem_fma_peak": [ctypes.c_int, dp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.efem_version.restype = ctypes.c_char_p
        _lib = L
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(2048)
    lib().efem_last_error(buf, 2048)
    return buf.value.decode(errors="replace")


def check(status):
    if status != OK:
        raise EfemError(status, last_error())


def fma_peak(fp32=False):
    """Measured CUDA-core FMA throughput of the current device, GFLOP/s (FP64,
    or FP32 with fp32=True): the compute roof of the element residual."""
    g = ctypes.c_double()
    check(lib().efem_fma_peak(1 if fp32 else 0, ctypes.byref(g)))
    return g.value


def default_options():
    o = Options()
    check(lib().efem_default_options(ctypes.byref(o)))
    return o


def _ptr(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def _vec_ptr(v):
    """Pointer of a float64 numpy array or a CUDA float64 torch tensor."""
    if hasattr(v, "data_ptr"):
        return ctypes.c_void_p(v.data_ptr())
    return ctypes.c_void_p(v.ctypes.data)


class Model:
    """One problem on one GPU (the C ABI's opaque handle)."""

    def __init__(self, handle):
        self.h = ctypes.c_void_p(handle) if not isinstance(handle, ctypes.c_void_p) else handle
        info = self.info()
        self.n_dof = info["n_dof"]
        self.n_free = info["n_free_nodes"]

    # ------------------------------------------------------------------ creation
    @classmethod
    def from_json(cls, path):
        h = ctypes.c_void_p()
        check(lib().efem_model_create_from_json(os.fsencode(path), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_arrays(cls, X, blocks, materials, loads, options=None):
        """X (n,3); blocks: list of (conn (ne,nen) 0-based, material ids or None);
        materials: dicts in the reference's JSON form; loads: list of
        ("fix", nodes) / ("force", nodes, [fx,fy,fz]) / ("pressure", faces, p) /
        ("dpressure", faces, [vx,vy,vz]) / ("gravity", [gx,gy,gz])."""
        keep = []
        X = np.ascontiguousarray(X, dtype=np.float64)
        keep.append(X)
        eb = (ElementBlock * max(1, len(blocks)))()
        for i, (conn, mids) in enumerate(blocks):
            conn = np.ascontiguousarray(conn, dtype=np.int32)
            keep.append(conn)
            eb[i].nen = conn.shape[1]
            eb[i].n_elem = conn.shape[0]
            eb[i].conn = _ptr(conn, ctypes.c_int)
            if mids is not None:
                mids = np.ascontiguousarray(mids, dtype=np.int32)
                keep.append(mids)
                eb[i].material_id = _ptr(mids, ctypes.c_int)
        mesh = MeshDesc(X.shape[0], _ptr(X), len(blocks), eb)
        tmap = {"neo_hookean": NEO_HOOKEAN, "mo_riv": MOONEY_RIVLIN, "yeoh": YEOH}
        mats = (Material * max(1, len(materials)))()
        for i, mj in enumerate(materials):
            mats[i] = Material(tmap[mj["type"]], int(mj.get("id", -1)), float(mj.get("C10", 0)),
                               float(mj.get("C01", 0)) if mj["type"] == "mo_riv" else 0.0,
                               float(mj.get("C20", 0)) if mj["type"] == "yeoh" else 0.0,
                               float(mj.get("C30", 0)) if mj["type"] == "yeoh" else 0.0,
                               float(mj.get("D1", 0)), float(mj.get("density", 0)))
        lds = (LoadDesc * max(1, len(loads)))()
        for i, ld in enumerate(loads):
            kind = ld[0]
            if kind in ("fix", "force"):
                nodes = np.ascontiguousarray(ld[1], dtype=np.int32)
                keep.append(nodes)
                lds[i].type = LOAD_FIX if kind == "fix" else LOAD_FORCE
                lds[i].n = nodes.shape[0]
                lds[i].nodes = _ptr(nodes, ctypes.c_int)
                if kind == "force":
                    for c in range(3):
                        lds[i].value[c] = float(ld[2][c])
            elif kind == "gravity":
                lds[i].type = LOAD_GRAVITY
                for c in range(3):
                    lds[i].value[c] = float(ld[1][c])
            else:
                faces = ld[1]
                ptr = np.zeros(len(faces) + 1, dtype=np.int32)
                ptr[1:] = np.cumsum([len(f) for f in faces])
                flat = np.ascontiguousarray(np.concatenate([np.asarray(f) for f in faces]) if faces else np.zeros(0),
                                            dtype=np.int32)
                keep += [ptr, flat]
                lds[i].type = LOAD_PRESSURE if kind == "pressure" else LOAD_DPRESSURE
                lds[i].n = len(faces)
                lds[i].nodes = _ptr(flat, ctypes.c_int)
                lds[i].face_ptr = _ptr(ptr, ctypes.c_int)
                vals = [float(ld[2]), 0.0, 0.0] if kind == "pressure" else [float(v) for v in ld[2]]
                for c in range(3):
                    lds[i].value[c] = vals[c]
        opts = options if options is not None else default_options()
        h = ctypes.c_void_p()
        check(lib().efem_model_create(ctypes.byref(mesh), mats, len(materials), lds, len(loads), ctypes.byref(opts),
                                      ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_case(cls, case, options=None):
        """Build from an ``efem_b200.meshgen.Case`` without writing files."""
        loads = [("fix", case.fix)]
        for value, nodes in case.force:
            loads.append(("force", nodes, value))
        for value, faces in case.pressure:
            if isinstance(value, (list, tuple, np.ndarray)):
                loads.append(("dpressure", faces, value))
            else:
                loads.append(("pressure", faces, value))
        g = case.analysis.get("gravity")
        if isinstance(g, str) and g in GRAVITY:
            loads.append(("gravity", GRAVITY[g]))
        opts = options if options is not None else default_options()
        opts.integration = 1 if case.integration == "reduced" else 0
        if isinstance(case.analysis.get("consistent_inertia"), bool):
            opts.consistent_inertia = int(case.analysis["consistent_inertia"])
        return cls.from_arrays(case.mesh.X, [(case.mesh.conn, case.mesh.mat)], case.materials, loads, opts)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().efem_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ options / info
    @property
    def options(self):
        o = Options()
        check(lib().efem_get_options(self.h, ctypes.byref(o)))
        return o

    def set_options(self, **kw):
        o = self.options
        for k, v in kw.items():
            setattr(o, k, v)
        check(lib().efem_set_options(self.h, ctypes.byref(o)))

    def info(self):
        i = ModelInfo()
        check(lib().efem_get_model_info(self.h, ctypes.byref(i)))
        return i.as_dict()

    def dof_map(self):
        out = np.zeros(self.n_free, dtype=np.int32)
        check(lib().efem_dof_map(self.h, _ptr(out, ctypes.c_int)))
        return out

    def external_load(self):
        """Nodal forces + M g per free DOF (host; no GPU needed)."""
        out = np.zeros(self.n_dof)
        check(lib().efem_external_load(self.h, _ptr(out)))
        return out

    # ------------------------------------------------------------------ hot path
    def residual(self, u, out=None):
        """R(u) for a host float64 array, or for CUDA float64 tensors when the
        model's ``device_ptrs`` option is set."""
        if out is None:
            out = np.zeros(self.n_dof) if not hasattr(u, "data_ptr") else u.new_zeros(self.n_dof)
        if not hasattr(u, "data_ptr"):
            u = np.ascontiguousarray(u, dtype=np.float64)
        check(lib().efem_residual(self.h, _vec_ptr(u), _vec_ptr(out)))
        return out

    def solve(self, u0=None):
        """L-BFGS solve from u0 (zeros by default); returns (u, info dict)."""
        if u0 is None:
            u = np.zeros(self.n_dof)
        elif hasattr(u0, "data_ptr"):
            u = u0
        else:
            u = np.array(u0, dtype=np.float64)
        info = SolveInfo()
        st = lib().efem_solve(self.h, _vec_ptr(u), ctypes.byref(info))
        if st not in (OK,):
            raise EfemError(st, last_error())
        return u, info.as_dict()

    def solve_trace(self):
        """Convergence trace of the last solve (options.trace > 0): a dict of
        arrays time_s, r_norm2, r_inf, step, r_evals, one entry per record
        (record 0: the initial residual; record i: after iteration i)."""
        n = ctypes.c_int(0)
        check(lib().efem_solve_trace(self.h, None, 0, ctypes.byref(n)))
        cap = min(n.value, self.options.trace)
        out = np.zeros((max(cap, 0), 5))
        if cap > 0:
            check(lib().efem_solve_trace(self.h, _ptr(out), cap, ctypes.byref(n)))
        return {"time_s": out[:, 0], "r_norm2": out[:, 1], "r_inf": out[:, 2], "step": out[:, 3],
                "r_evals": out[:, 4].astype(np.int64), "n_records": n.value}

    # ------------------------------------------------------------------ sensitivities
    def _vec(self, x):
        if hasattr(x, "data_ptr"):
            return x
        return np.ascontiguousarray(x, dtype=np.float64)

    def _out_like(self, x):
        if hasattr(x, "data_ptr"):
            import torch
            return torch.empty(self.n_dof, dtype=torch.float64, device=x.device)
        return np.zeros(self.n_dof)

    def hvp(self, u, v, transpose=False):
        """K(u) v (K(u)^T v with transpose=True), the true tangent at u."""
        u, v = self._vec(u), self._vec(v)
        out = self._out_like(u)
        f = lib().efem_hvp_transpose if transpose else lib().efem_hvp
        check(f(self.h, _vec_ptr(u), _vec_ptr(v), _vec_ptr(out)))
        return out

    def param_derivative(self, u, k):
        """dR/dtheta_k at u (parameter order: efem_residual_param_derivative)."""
        u = self._vec(u)
        out = self._out_like(u)
        check(lib().efem_residual_param_derivative(self.h, _vec_ptr(u), int(k), _vec_ptr(out)))
        return out

    def write_vtk(self, path, u=None):
        """Legacy ASCII VTK of the mesh at X + u (u None: reference configuration)."""
        uu = None if u is None else self._vec(u)
        check(lib().efem_write_vtk(self.h, _vec_ptr(uu) if uu is not None else None, str(path).encode()))

    def strain_energy(self, u):
        """Stored strain energy at u, summed in FP64."""
        u = self._vec(u)
        e = ctypes.c_double()
        check(lib().efem_strain_energy(self.h, _vec_ptr(u), ctypes.byref(e)))
        return e.value

    @property
    def n_params(self):
        return self.info()["n_params"]

    def adjoint(self, u, dJdu, want_lambda=False):
        """dJ/dtheta at the equilibrium u for the objective gradient dJ/du;
        returns (dJdtheta, lambda or None, info dict)."""
        u, g = self._vec(u), self._vec(dJdu)
        out = np.zeros(self.n_params)
        lam = self._out_like(u) if want_lambda else None
        info = AdjointInfo()
        check(lib().efem_adjoint(self.h, _vec_ptr(u), _vec_ptr(g), _ptr(out),
                                 _vec_ptr(lam) if lam is not None else None, ctypes.byref(info)))
        return out, lam, info.as_dict()

    def approx_jacobian_csr(self):
        nnz = ctypes.c_longlong()
        check(lib().efem_approx_jacobian_csr(self.h, ctypes.byref(nnz), None, None, None))
        rp = np.zeros(self.n_free + 1, dtype=np.int32)
        ci = np.zeros(nnz.value, dtype=np.int32)
        v = np.zeros(nnz.value)
        check(lib().efem_approx_jacobian_csr(self.h, ctypes.byref(nnz), _ptr(rp, ctypes.c_int), _ptr(ci, ctypes.c_int),
                                             _ptr(v)))
        return rp, ci, v

    def precond_apply(self, v):
        """H0 v (in place for a CUDA tensor when device_ptrs is set)."""
        if not hasattr(v, "data_ptr"):
            v = np.array(v, dtype=np.float64)
        check(lib().efem_precond_apply(self.h, _vec_ptr(v)))
        return v

    def set_stream(self, cuda_stream_handle):
        """Run on the caller's CUDA stream (an integer cudaStream_t, e.g.
        torch.cuda.current_stream().cuda_stream); None for the model's own."""
        check(lib().efem_set_stream(self.h, ctypes.c_void_p(cuda_stream_handle)))


def batch_solve(models, us=None, max_threads=0):
    """Solve independent models concurrently (efem_batch_solve).  us: initial
    solutions (zeros by default), numpy arrays or CUDA tensors per each
    model's device_ptrs option; solved in place.  Returns (us, info dicts)."""
    n = len(models)
    if us is None:
        us = [np.zeros(m.n_dof) for m in models]
    hs = (ctypes.c_void_p * n)(*[m.h.value for m in models])
    ptrs = (ctypes.c_void_p * n)(*[_vec_ptr(u).value for u in us])
    infos = (SolveInfo * n)()
    check(lib().efem_batch_solve(hs, n, ptrs, infos, int(max_threads)))
    return us, [infos[i].as_dict() for i in range(n)]


class Simulator:
    """The reference's JSON-driven call: ``initial(path)`` then ``start()``."""

    def __init__(self):
        self.model = None
        self.u = None
        self.result = None

    def initial(self, config_file_path):
        self.model = Model.from_json(config_file_path)
        return self

    def start(self):
        self.u, self.result = self.model.solve()
        return self.result
