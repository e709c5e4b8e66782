"""Benchmark: L-BFGS iterations/s and time-to-converge of the hyperelastic solve.

Workload (one step = the first 32 L-BFGS iterations of the reference's
JSON-driven solve from u = 0, criterion ||r||_inf <= 1e-6): the C3D8 beam, 0.2 x 0.04 x 0.04 m on an
80 x 16 x 16 hexahedral grid (20 480 elements, 23 409 nodes, 69 360 DOF),
Mooney-Rivlin C10 = 80 kPa, C01 = 20 kPa, D1 = 1e-6, x = 0 fixed, nodal force
[0, 0, -0.5] N on each of the 289 end-face nodes; FP64 element kernels (or the
mixed FP32 path with --precision mixed).  Synthetic, seeded mesh in the
reference's own file formats (efem_b200.meshgen).

The reference's solve of this beam does not converge: at its seventh
iteration the line search accepts a trial with elements turned inside out
(its laws stay finite there, J^{-2/3} taken as (J^2)^{-1/3}) and ||r||
grows without bound, every later iteration exhausting the 20 line-search
trials.  This library follows the same record (``parity`` below), so a step
is a fixed count of iterations on that path, the same work on both arms;
time-to-converge is measured on the cap (``mixed_vs_fp64``), which converges
in 91 iterations here and in the reference.

Each timed step includes the per-solve numeric factorisation of the
approximate Jacobian (as LBFGSSolver::solve does once per solve); the mesh
set-up (element tables, symbolic analysis of the factor) happens once, before
the warm-up steps.

After the timed region the default line also carries, on one GPU, the rest
of the metric: ``parity`` (||r||_2 after each of the first line searches
against the reference's own record of this solve, a committed fixture),
``mixed_vs_fp64`` (the C3D20R cylinder cap's time-to-converge in mixed
precision and in FP64, each solution's error against the reference) and
``adjoint`` / ``adjoint_ms`` (the finger's gradient time); --no-extras skips
the last two.

--gpus N: N independent replicas (one process per GPU, the solve does not
shard); value = iterations of all ranks / max-over-ranks time.
--impl reference: the reference's own CPU solver (compiled from its sources in
oracle/_ref), timed on the host cores on bounded samples of the same solve.

--workload batch: the batched time-to-solution of 256 uneven C3D4 beams
(efem_b200.meshgen.batch_beams, 2.65 M elements in all), mixed precision, as
one union model in one iteration graph (efem_batch_solve), next to the same
batch in FP64 and to the plain FP64 path solving the models one after
another.

--workload cap: time-to-converge of the closed cylinder cap (C3D20 reduced
integration, 9088 elements, 10 kPa cavity pressure) in mixed precision next
to the FP64 path, with the mixed solution's error against FP64 converged to
1e-10.

--workload finger-adjoint: the adjoint gradient time instead (ms per
gradient): the pneumatic finger, 50 688 C3D10 Yeoh elements with 30 kPa on
its 8 chamber walls, J = u_z of the tip node, dJ/dtheta for every material
constant and the pressure, at the converged equilibrium.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "L-BFGS iters/s (first 32 iterations of the reference's solve, C3D8 MR beam 20480 el)"
# iterations per step: the reference's solve of the beam does not converge.  32
# is as far as the reference arm's samples reach (iterations 9-32); further
# along, ||r|| (about 1e93 N by then) can overflow and end the solve as
# non-finite, in the reference as here, at a point that varies with rounding
BEAM_ITERS = 32
UNIT = "iters/s"


def workload_case():
    from efem_b200 import meshgen as mg
    return mg.cantilever_c3d8_force()


def config_block(precision, n):
    return {"workload": "C3D8 Mooney-Rivlin cantilever, 80x16x16 hex (20480 el, 69360 DOF), tip force, "
                        "residual 1e-6, the first 32 L-BFGS iterations of the solve from u = 0 per step "
                        "(the reference's solve of this beam does not converge)",
            "precision": precision, "elements": 20480, "dof": 69360, "replicas": n,
            "parallelism": f"replicas{n}", "l2": "flushed (256 MB write) before every step"}


# --------------------------------------------------------------------------- replicas
def combine_ranks(ms, units, world, device="cpu"):
    """Whole-job figures over replicas: (the slowest rank's time, the units of
    all ranks).  Every rank calls it, in the same order (two all-reduces)."""
    if world <= 1:
        return float(ms), float(units)
    import torch
    import torch.distributed as dist
    tm = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    tu = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(tm, op=dist.ReduceOp.MAX)
    dist.all_reduce(tu, op=dist.ReduceOp.SUM)
    return float(tm[0]), float(tu[0])


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for ln in open(self.path):
                p = [x.strip() for x in ln.split(",")]
                if len(p) >= 9 and p[1].isdigit():
                    rows.append(p)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = np.array([float(r[1]) for r in rows])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


# --------------------------------------------------------------------------- reference arm
def reference_sample(steps, warmup, ipstep=8):
    """The reference's own solver on bounded samples of the workload: one-time
    factorisation, then `warmup` + `steps` steps of `ipstep` L-BFGS iterations.
    Returns (iters/s over the timed steps, details).  The reference's time per
    iteration grows along the solve (0.21 s per iteration at iterations 3-6,
    0.7-0.9 s from iteration 7 on this beam, where its line search starts to
    use all 20 trials), so a step spans several iterations."""
    ref = os.path.join(ROOT, "oracle", "_ref", "efem_ref")
    if not os.path.exists(ref):
        return None, {"why": "oracle/_ref/efem_ref is not built"}
    case = workload_case()
    with tempfile.TemporaryDirectory() as td:
        cfg = case.write(td)
        t0 = time.time()
        res = subprocess.run([ref, "bench", cfg, str(ipstep), str(warmup), str(steps)], capture_output=True,
                             text=True, timeout=3600)
        wall = time.time() - t0
    if res.returncode != 0:
        return None, {"why": res.stderr[-300:]}
    meta = json.loads(res.stdout.strip().splitlines()[-1])
    st = meta["step_s"]
    if not st:
        return None, {"why": "reference converged inside the warm-up"}
    ips = ipstep * len(st) / sum(st)
    meta.update(wall_s=wall)
    return ips, meta


def reference_batch_sample(cases, n_proc, ipstep=8, warmup=1, steps=2):
    """The reference's own solver on n_proc batch models at once, one process
    per host core (the reference solves one problem per process): each one
    factors once (excluded), then runs `warmup` + `steps` steps of `ipstep`
    L-BFGS iterations.  Returns (aggregate iters/s over the timed steps, the
    models sampled, details)."""
    ref = os.path.join(ROOT, "oracle", "_ref", "efem_ref")
    if not os.path.exists(ref):
        return None, 0, {"why": "oracle/_ref/efem_ref is not built"}
    with tempfile.TemporaryDirectory() as td:
        procs = []
        for i, c in enumerate(cases[:n_proc]):
            cfg = c.write(os.path.join(td, f"m{i}"))
            procs.append(subprocess.Popen([ref, "bench", cfg, str(ipstep), str(warmup), str(steps)],
                                          stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
        rate, used = 0.0, 0
        for p in procs:
            out, err = p.communicate(timeout=3600)
            if p.returncode != 0:
                return None, 0, {"why": err[-300:]}
            st = json.loads(out.strip().splitlines()[-1])["step_s"]
            if st:  # a model that converged inside the warm-up adds nothing
                rate += ipstep * len(st) / sum(st)
                used += 1
    return rate, used, {}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ips, meta = reference_sample(args.steps, args.warmup)
    if ips is None:
        print(json.dumps({"impl": "reference", "unavailable": meta.get("why", "reference failed")}))
        return
    cores = 1
    line = {"impl": "reference", "metric": METRIC, "value": ips, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * meta["iters_per_step"] / ips,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_block("fp64", 1),
            "cpu_baseline": {"value": ips, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"reference solver (oracle/_ref, unmodified sources, single-threaded as built "
                                       f"upstream) on the same C3D8 beam: one-time approximate-Jacobian "
                                       f"factorisation ({meta['factor_s']:.1f} s, outside the timed steps), then "
                                       f"{args.steps} timed steps of {meta['iters_per_step']} L-BFGS iterations"},
            "e2e": {"value": ips, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_factor_s": meta["factor_s"]}
    print(json.dumps(line))


# --------------------------------------------------------------------------- adjoint gradient
def measure_adjoint(steps, warmup, stream):
    """Adjoint gradient time on the pneumatic finger: returns a dict with the
    mean device time per gradient (CUDA events on the model's stream), the
    end-to-end time through host buffers, the GMRES iterations and the
    whole adjoint solve's HBM roofline."""
    import torch
    from efem_b200 import api, meshgen as mg, profiling
    case, tip = mg.finger_c3d10()
    opts = api.default_options()
    opts.max_iterations = 20000  # a bound for the equilibrium solve
    t_setup = time.time()
    model = api.Model.from_case(case, opts)
    api.check(api.lib().efem_set_stream(model.h, api.ctypes.c_void_p(stream.cuda_stream)))
    model.set_options(device_ptrs=1)
    u = torch.zeros(model.n_dof, dtype=torch.float64, device="cuda")
    _, sinfo = model.solve(u)
    setup_s = time.time() - t_setup
    dnode = int(np.nonzero(model.dof_map() == tip)[0][0])
    g = torch.zeros(model.n_dof, dtype=torch.float64, device="cuda")
    g[3 * dnode + 2] = 1.0
    for _ in range(warmup):
        model.adjoint(u, g)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    infos = []
    for a, b in ev:
        a.record(stream)
        grad, _, info = model.adjoint(u, g)
        b.record(stream)
        infos.append(info)
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in ev]
    # end to end with host buffers: u and dJ/du copied in, dJ/dtheta out
    model.set_options(device_ptrs=0)
    u_h = torch.empty(model.n_dof, dtype=torch.float64).pin_memory()
    u_h.copy_(u.cpu())
    g_h = torch.zeros(model.n_dof, dtype=torch.float64).pin_memory()
    g_h[3 * dnode + 2] = 1.0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    model.adjoint(u_h.numpy(), g_h.numpy())
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    info = model.info()
    # whole adjoint solve against HBM: its algorithmic bytes (the library's
    # count per Krylov iteration) over its time (host clock around the solve,
    # ended by a stream synchronisation)
    hbm, hbm_kind = profiling.hbm_peak()
    solve_s = float(np.mean([i["ms_solve"] for i in infos])) / 1000.0
    nbytes = float(np.mean([i["solve_bytes"] for i in infos]))
    achieved = nbytes / solve_s / 1e9
    out = {"ms": float(np.mean(ms)), "ms_all": ms, "e2e_ms": e2e_ms, "dof": model.n_dof,
           "elements": info["n_elements"], "parameters": info["n_params"],
           "gmres_iterations": float(np.mean([i["iterations"] for i in infos])),
           "adjoint_solve_ms": float(np.mean([i["ms_solve"] for i in infos])),
           "parameter_sensitivities_ms": float(np.mean([i["ms_params"] for i in infos])),
           "adjoint_tolerance": model.options.adjoint_tolerance,
           "equilibrium_solve": {"niter": sinfo["niter"], "ms": sinfo["ms_total"], "r_inf": sinfo["r_inf"]},
           "setup_s": setup_s, "gpu_launches": int(sum(i["n_kernel_launches"] for i in infos)),
           "h2d_bytes": 2 * 8 * model.n_dof, "d2h_bytes": 8 * info["n_params"],
           "roofline": {"kernel": "adjoint solve (GMRES: k_solve H0, transpose tangent, Gram-Schmidt)",
                        "bound": "hbm", "achieved": achieved, "peak": hbm, "peak_source": hbm_kind, "unit": "GB/s",
                        "frac": achieved / hbm, "traffic": None, "algorithmic_bytes_per_gradient": nbytes}}
    model.close()
    return out


def run_adjoint_bench(args):
    """Adjoint gradient time on the pneumatic finger (one GPU)."""
    import torch
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    with ClockSampler(0) as clocks:
        a = measure_adjoint(args.steps, args.warmup, stream)
    line = {"metric": "adjoint gradient time (dJ/dtheta, C3D10 Yeoh finger 50688 el)", "value": a["ms"],
            "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": a["ms"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded structured mesh in the reference's input format)",
            "config": {"workload": "pneumatic finger 80x15x15 mm, 8 chambers, 50688 C3D10 (Yeoh), 30 kPa on the "
                                   "chamber walls, J = u_z of the tip node, gradient w.r.t. all material constants "
                                   "and the pressure at the converged equilibrium", "dof": a["dof"],
                       "elements": a["elements"], "parameters": a["parameters"],
                       "adjoint_tolerance": a["adjoint_tolerance"]},
            "gmres_iterations": a["gmres_iterations"], "adjoint_solve_ms": a["adjoint_solve_ms"],
            "parameter_sensitivities_ms": a["parameter_sensitivities_ms"],
            "equilibrium_solve": a["equilibrium_solve"], "setup_s": a["setup_s"],
            "e2e": {"value": a["e2e_ms"], "unit": "ms", "h2d_bytes_per_step": a["h2d_bytes"],
                    "d2h_bytes_per_step": a["d2h_bytes"]},
            "gpu_launches": a["gpu_launches"], "roofline": a["roofline"], "clocks": clocks.summary()}
    print(json.dumps(line))


# --------------------------------------------------------------------------- C3D20R cap, mixed vs FP64
def reference_fixture(name):
    """The reference's converged displacement of a generated benchmark mesh
    (tests/golden/config_<name>.npz, made by tests/golden/make_golden.py from
    the reference compiled in oracle/_ref), or None."""
    path = os.path.join(ROOT, "tests", "golden", f"config_{name}.npz")
    if not os.path.exists(path):
        return None
    d = np.load(path, allow_pickle=False)
    return {"u": d["u_solve"].astype(np.float64), "meta": json.loads(str(d["solve_meta"])),
            "epsilon": float(d["epsilon"])}


BEAM_RECORD_PINNED = 8  # records 0-7: before the divergent iterations amplify rounding


def beam_solve(model, u):
    """One step's solve of the beam: its info dict.  The reference's path on
    this beam can end non-finite at an iteration that moves with rounding
    (then the solve stops with EFEM_ERR_NAN and u zeroed, as the reference's
    Integrator::integral does); the iterations done up to there count."""
    from efem_b200 import api
    import ctypes
    info = api.SolveInfo()
    st = api.lib().efem_solve(model.h, api._vec_ptr(u), ctypes.byref(info))
    if st not in (api.OK, api.ERR_NAN):
        raise api.EfemError(st, api.last_error())
    d = info.as_dict()
    d["non_finite"] = st == api.ERR_NAN
    return d


def beam_record_parity(model):
    """||r||_2 after the initial residual and after each line search of a
    traced solve of the beam, against the reference's own record of the same
    solve (tests/golden/config_beam_c3d8_mr_force_record.npz, made by
    tests/golden/make_golden.py from the reference compiled in oracle/_ref).
    The first eight records agree to rounding; from the ninth on both solves
    have left every bound (the reference's passes 1e9 N), each along its own
    rounding, as the reference and its C restatement do as well."""
    path = os.path.join(ROOT, "tests", "golden", "config_beam_c3d8_mr_force_record.npz")
    if not os.path.exists(path):
        return None
    d = np.load(path, allow_pickle=False)
    ref = d["r_norm2"]
    n = len(ref)
    model.set_options(device_ptrs=0, trace=n, max_iterations=n - 1)
    beam_solve(model, np.zeros(model.n_dof))
    tr = model.solve_trace()["r_norm2"]
    model.set_options(trace=0, max_iterations=BEAM_ITERS)
    k = min(len(tr), n)
    rel = np.abs(tr[:k] - ref[:k]) / ref[:k]
    return {"records": int(k), "max_rel_diff_first_8": float(rel[:BEAM_RECORD_PINNED].max()),
            "r_norm2": [float(x) for x in tr[:k]], "reference_r_norm2": [float(x) for x in ref[:k]],
            "reference": "the reference's LBFGSSolver::solve of the same mesh (oracle/_ref): its benchmark "
                         "record, which does not converge"}


def measure_cap(steps, warmup, stream):
    """Time-to-converge of the C3D20R cylinder cap in mixed precision and in
    FP64 (same stream, L2 flushed before every solve), each solution's error
    against the reference's own FP64 solve of the same mesh and against this
    library's FP64 solve converged to 1e-10 N."""
    import torch
    from efem_b200 import api, meshgen as mg
    case = mg.cylinder_cap_c3d20()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def build(precision, criterion=1e-6):
        o = api.default_options()
        o.precision = precision
        o.residual_criterion = criterion
        o.max_iterations = 20000  # a bound; both precisions converge in a few hundred iterations
        m = api.Model.from_case(case, o)
        api.check(api.lib().efem_set_stream(m.h, api.ctypes.c_void_p(stream.cuda_stream)))
        m.set_options(device_ptrs=1)
        return m, torch.zeros(m.n_dof, dtype=torch.float64, device="cuda")

    def timed(m, u, n):
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        infos = []
        for k, (a, b) in enumerate(ev):
            flush.fill_(float(k))
            u.zero_()
            a.record(stream)
            infos.append(m.solve(u)[1])
            b.record(stream)
        torch.cuda.synchronize()
        return float(np.mean([a.elapsed_time(b) for a, b in ev])), infos

    t0 = time.time()
    m32, u32 = build(api.MIXED)
    m64, u64 = build(api.FP64)
    for _ in range(max(1, warmup)):
        timed(m32, u32, 1)
        timed(m64, u64, 1)
    setup_s = time.time() - t0
    ms32, i32 = timed(m32, u32, steps)
    ms64, i64 = timed(m64, u64, steps)
    mref, uref = build(api.FP64, 1e-10)
    mref.set_options(max_iterations=50000)
    _, iref = mref.solve(uref)
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))  # noqa: E731
    r64_at_mixed = float(m64.residual(u32).abs().max())  # device_ptrs: CUDA tensors in and out
    fx = reference_fixture("cap_c3d20r_nh_pressure")
    vs_ref = {}
    if fx is not None:
        ur = torch.from_numpy(fx["u"]).cuda()
        vs_ref = {"mixed": rel(u32, ur), "fp64": rel(u64, ur), "fp64_1e-10": rel(uref, ur),
                  "reference_niter": fx["meta"]["niter"], "reference_epsilon": fx["epsilon"]}
    info = m32.info()
    n32 = max(1.0, float(np.mean([i["niter"] for i in i32])))
    n64 = max(1.0, float(np.mean([i["niter"] for i in i64])))
    out = {"elements": info["n_elements"], "dof": m32.n_dof, "faces": info["n_faces"],
           "mixed": {"ms": ms32, "niter": n32, "r_inf": i32[-1]["r_inf"],
                     "refined": bool(i32[-1]["flags"] & api.SOLVE_REFINED),
                     "rel_l2_vs_fp64_1e-10": rel(u32, uref), "fp64_residual_at_mixed_solution": r64_at_mixed,
                     "ms_per_iteration": ms32 / n32},
           "fp64": {"ms": ms64, "niter": n64, "r_inf": i64[-1]["r_inf"],
                    "rel_l2_vs_fp64_1e-10": rel(u64, uref), "ms_per_iteration": ms64 / n64},
           "fp64_over_mixed_time": ms64 / ms32,
           "rel_l2_vs_reference": vs_ref,
           "fp64_1e-10_solution": {"niter": iref["niter"], "r_inf": iref["r_inf"]},
           "setup_s": setup_s}
    for m in (m32, m64, mref):
        m.close()
    return out


CAP_WORKLOAD = ("hollow cylinder ri 20 mm, ro 25 mm, h 30 mm, 5 mm top plate; 64x4x24 shell + butterfly plate; "
                "C3D20 reduced integration; NH C10 114 kPa, D1 1e-6; bottom fixed; 10 kPa follower pressure on the "
                "cavity walls; residual 1e-6")


def run_cap_bench(args):
    """Time-to-converge of the C3D20R cylinder cap, mixed precision vs FP64 (one GPU)."""
    import torch
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    with ClockSampler(0) as clocks:
        c = measure_cap(args.steps, args.warmup, stream)
    line = {"metric": "time-to-converge, mixed precision (C3D20R cylinder cap, 9088 el)", "value": c["mixed"]["ms"],
            "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": c["mixed"]["ms"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded structured mesh in the reference's input format)",
            "config": {"workload": CAP_WORKLOAD, "elements": c["elements"], "dof": c["dof"], "faces": c["faces"],
                       "l2": "flushed (256 MB write) before every solve"},
            **{k: c[k] for k in ("mixed", "fp64", "fp64_over_mixed_time", "rel_l2_vs_reference",
                                 "fp64_1e-10_solution", "setup_s")},
            "clocks": clocks.summary()}
    print(json.dumps(line))


# --------------------------------------------------------------------------- batched solves
def run_batch_bench(args):
    """Mixed-precision batched solves of 256 uneven beams (one union model, one
    iteration graph) next to the same batch in FP64 and to the plain FP64
    path solving the models one after another."""
    import torch
    from efem_b200 import api, meshgen as mg
    torch.cuda.set_device(0)
    t0 = time.time()
    cases = mg.batch_beams()
    gen_s = time.time() - t0

    def build(precision, criterion=1e-6):
        ms, us = [], []
        for c in cases:
            o = api.default_options()
            o.precision = precision
            o.residual_criterion = criterion
            o.max_iterations = 50000  # a bound for the batch; every beam converges well before it
            m = api.Model.from_case(c, o)
            m.set_options(device_ptrs=1)
            ms.append(m)
            us.append(torch.zeros(m.n_dof, dtype=torch.float64, device="cuda"))
        return ms, us

    def run_batch(ms, us):
        for u in us:
            u.zero_()
        torch.cuda.synchronize()
        a = time.perf_counter()
        _, infos = api.batch_solve(ms, us)
        torch.cuda.synchronize()
        return time.perf_counter() - a, infos

    def run_sequential(ms, us):
        for u in us:
            u.zero_()
        torch.cuda.synchronize()
        a = time.perf_counter()
        infos = [m.solve(u)[1] for m, u in zip(ms, us)]
        torch.cuda.synchronize()
        return time.perf_counter() - a, infos

    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))  # noqa: E731
    t0 = time.time()
    m32, u32 = build(api.MIXED)
    m64, u64 = build(api.FP64)
    build_s = time.time() - t0
    t0 = time.time()
    run_batch(m32, u32)          # first calls: union set-up, symbolic analyses, graph captures
    run_batch(m64, u64)
    run_sequential(m64, u64)
    setup_s = time.time() - t0
    for _ in range(max(0, args.warmup - 1)):
        run_batch(m32, u32)
    times, infos = [], None
    with ClockSampler(0) as clocks:
        for _ in range(args.steps):
            t, infos = run_batch(m32, u32)
            times.append(t)
        t64b, infos64b = run_batch(m64, u64)
        u64b = [u.clone() for u in u64]
        t64, infos64 = run_sequential(m64, u64)
    # accuracy against FP64 solves converged to 1e-10, at the reference's 1e-6 N and at 1e-9 N
    mref, uref = build(api.FP64, 1e-10)
    api.batch_solve(mref, uref)
    err = max(rel(a, b) for a, b in zip(u32, uref))
    err64 = max(rel(a, b) for a, b in zip(u64, uref))
    for m in m32:
        m.set_options(residual_criterion=1e-9)
    t_tight, infos_tight = run_batch(m32, u32)
    err_tight = max(rel(a, b) for a, b in zip(u32, uref))
    iters = sum(i["niter"] for i in infos)
    conv = sum(1 for i in infos if i["flags"] & api.SOLVE_CONVERGED)
    t = float(np.mean(times))
    line = {"metric": "batched time-to-solution, mixed precision (256 uneven C3D4 beams, 2.65M el)", "value": t,
            "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded: efem_b200.meshgen.batch_beams(seed=20261203))",
            "config": {"workload": "256 C3D4 cantilevers, L 50-200 mm, section 10-30 mm, h 2-5 mm (648-39930 "
                                   "elements each), NH or MR, C10 5e4-5e5 Pa, end pressure 1-20 kPa capped at half "
                                   "the Euler buckling load, residual 1e-6",
                       "models": len(cases), "elements": int(sum(c.mesh.conn.shape[0] for c in cases)),
                       "batching": "one union model: one element-kernel launch per element type, one forest "
                                   "factorisation and triangular solve, segmented L-BFGS kernels, one CUDA graph "
                                   "of the iteration loop (efem_batch_solve)",
                       "timing": "host clock around the whole batch, device synchronised before and after"},
            "union": all(bool(i["flags"] & api.SOLVE_BATCHED) for i in infos),
            "batch_iterations": iters, "iterations_per_s": iters / t, "converged": conv,
            "max_iterations_of_a_member": max(i["niter"] for i in infos),
            "refined_members": sum(1 for i in infos if i["flags"] & api.SOLVE_REFINED),
            "fp64_batched_s": t64b, "mixed_speedup_vs_fp64_batched": t64b / t,
            "fp64_sequential_s": t64, "speedup_vs_fp64_sequential": t64 / t,
            "fp64_sequential_iterations": sum(i["niter"] for i in infos64),
            "fp64_batched_vs_sequential_max_rel_l2": max(rel(a, b) for a, b in zip(u64b, u64)),
            "mixed_vs_fp64_max_rel_l2": err,
            "fp64_at_1e-6_vs_fp64_max_rel_l2": err64,
            "at_1e-9": {"mixed_s": t_tight, "mixed_vs_fp64_max_rel_l2": err_tight,
                        "converged": sum(1 for i in infos_tight if i["flags"] & api.SOLVE_CONVERGED)},
            "accuracy_reference": "FP64 solves of the same models converged to residual 1e-10",
            "generate_s": gen_s, "build_s": build_s, "setup_s": setup_s,
            "clocks": clocks.summary()}
    if not args.no_cpu_baseline:
        cores = min(len(cases), os.cpu_count() or 1)
        rate, used, meta = reference_batch_sample(cases, cores)
        if rate is not None:
            line["cpu_baseline"] = {"value": rate, "unit": "iters/s (aggregate)", "cores": cores, "kind": "reference",
                                    "sample": f"reference solver (oracle/_ref), one process per host core on the "
                                              f"first {cores} batch models at once: one factorisation each "
                                              f"(excluded), then 2 timed steps of 8 L-BFGS iterations; "
                                              f"{used} models timed; compare with iterations_per_s"}
    print(json.dumps(line))


# --------------------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="efem_b200", choices=["efem_b200", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-vs-FP64 (cap) and adjoint (finger) blocks of the default line")
    ap.add_argument("--host-loop", action="store_true",
                    help="drive the L-BFGS iterations from the host (same kernels; for launch-list profiling)")
    ap.add_argument("--workload", default="beam", choices=["beam", "finger-adjoint", "batch", "cap"])
    args = ap.parse_args()
    if args.impl == "reference":
        if args.workload != "beam":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no adjoint or tangent"}))
            return
        return run_reference_arm(args)
    if args.workload == "finger-adjoint":
        return run_adjoint_bench(args)
    if args.workload == "batch":
        return run_batch_bench(args)
    if args.workload == "cap":
        return run_cap_bench(args)

    import torch
    import torch.distributed as dist
    from efem_b200 import api

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    case = workload_case()
    opts = api.default_options()
    opts.precision = api.MIXED if args.precision == "mixed" else api.FP64
    opts.device = local
    opts.host_loop = 1 if args.host_loop else 0
    opts.max_iterations = BEAM_ITERS
    t_setup = time.time()
    model = api.Model.from_case(case, opts)
    stream = torch.cuda.current_stream()
    api.check(api.lib().efem_set_stream(model.h, api.ctypes.c_void_p(stream.cuda_stream)))
    model.set_options(device_ptrs=1)
    u = torch.zeros(model.n_dof, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def one_solve():
        u.zero_()
        return beam_solve(model, u)

    first = one_solve()  # also builds the symbolic factor analysis
    setup_s = time.time() - t_setup
    for _ in range(args.warmup):
        one_solve()
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    infos = []
    with ClockSampler(local) as clocks:
        barrier()
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            infos.append(one_solve())
            ev[k][1].record(stream)
        barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    iters = sum(i["niter"] for i in infos)
    total_ms_max, iters_all = combine_ranks(total_ms, iters, world, "cuda")
    value = iters_all / (total_ms_max / 1000.0)

    # ---- end to end through the C ABI with host buffers (pinned host input / output)
    model.set_options(device_ptrs=0)
    u_host = torch.zeros(model.n_dof, dtype=torch.float64).pin_memory().numpy()
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(max(1, args.steps // 2))]
    e2e_iters = 0
    barrier()
    for a, b in e2e_ev:
        u_host[:] = 0.0
        a.record(stream)
        info = beam_solve(model, u_host)
        b.record(stream)
        e2e_iters += info["niter"]
    barrier()
    e2e_ms = sum(a.elapsed_time(b) for a, b in e2e_ev)
    e2e_ms_max, e2e_iters_all = combine_ranks(e2e_ms, e2e_iters, world, "cuda")
    e2e_value = e2e_iters_all / (e2e_ms_max / 1000.0)

    # ---- roofline of the dominant kernel, measured live on the model's stream
    from efem_b200 import profiling
    roof, launches = profiling.roofline_report(model, infos)
    fp32_res = args.precision == "mixed"
    roof["residual_compute"] = profiling.residual_compute_roof(
        model, infos, api.fma_peak(fp32=fp32_res), "FP32" if fp32_res else "FP64")

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded structured mesh in the reference's input format)",
            "config": config_block(args.precision, world),
            "iterations_per_step": iters / args.steps,
            "steps_ended_non_finite": sum(1 for i in infos if i.get("non_finite")), "residual_evals_per_solve": sum(i["n_residual_evals"] for i in infos) / args.steps,
            "final_r_inf": infos[-1]["r_inf"], "u_inf": infos[-1]["u_inf"],
            "converged": all(bool(i["flags"] & api.SOLVE_CONVERGED) for i in infos),
            "programmatic_dependent_launch": all(bool(i["flags"] & api.SOLVE_PDL) for i in infos),
            "factor_ms": float(np.mean([i["ms_factor"] for i in infos])),
            "setup_s": setup_s,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * model.n_dof,
                    "d2h_bytes_per_step": 8 * model.n_dof},
            "gpu_launches": int(launches * args.steps),
            "roofline": roof,
            "clocks": clocks.summary()}
    # ---- parity: ||r||_2 after each line search against the reference's own record of this solve
    line["parity"] = beam_record_parity(model)
    # ---- the rest of the metric, after the timed region: mixed vs FP64 (C3D20R cap) and the adjoint gradient
    if rank == 0 and world == 1 and not args.no_extras:
        c = measure_cap(3, 1, stream)
        line["mixed_vs_fp64"] = {"workload": CAP_WORKLOAD, **c}
        a = measure_adjoint(3, 1, stream)
        line["adjoint"] = {"workload": "pneumatic finger, 50688 C3D10 Yeoh, 30 kPa chambers, dJ/dtheta of the "
                                       "tip node's u_z for every material constant and the pressure", **a}
        line["adjoint_ms"] = a["ms"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ips, meta = reference_sample(steps=3, warmup=1)
        if ips is not None:
            line["cpu_baseline"] = {"value": ips, "unit": UNIT, "cores": 1, "kind": "reference",
                                    "sample": f"reference solver (oracle/_ref) on the same beam: approximate-Jacobian "
                                              f"factorisation once ({meta['factor_s']:.1f} s, excluded), then 3 timed "
                                              f"steps of {meta['iters_per_step']} L-BFGS iterations; single-threaded"}
    if rank == 0:
        print(json.dumps(line))
    model.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
