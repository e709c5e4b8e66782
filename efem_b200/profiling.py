"""Roofline bookkeeping for bench.py.

The solve reports device time per phase, summed on the device from the
GPU's global timer at the start and end of every residual evaluation and
every H0 application (efem_solve_info.ms_residual / ms_precond; the first H0
application of a solve is timed with CUDA events).  From those and the
algorithmic byte counts the library reports (efem_model_info), this module
picks the dominant kernel group of the timed solves and forms

    achieved = algorithmic bytes per launch / mean launch duration
    frac     = achieved / measured HBM copy bandwidth (MEASURED_PEAKS.json)

Algorithmic bytes per launch:
  residual   every input read once (connectivity, material index, V_e,
             J0^{-1} per Gauss point, u, f_ext) and r written once
  H0 apply   nnz(L) factor entries read in each sweep: the forward sweep
             reads L_JJ^{-1} (lower triangle) and W = L_RJ L_JJ^{-1}, the
             backward sweep their transposes; plus five passes over the
             3-component vectors (right-hand side, y written and read, x
             gathered and written); the fronts' update vectors (a few per cent
             of the total) are not counted
"""
from __future__ import annotations

import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def measured_traffic(kernel_group):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum of
    one ncu capture) from profiles/traffic.json, if present."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get(kernel_group)
    except Exception:
        return None


def residual_compute_roof(model, infos, fma_gflops, fma_kind):
    """The element residual against its own roofs: achieved GFLOP/s (the
    library's algorithmic flop count per evaluation over the mean device time
    of one evaluation) and the attainable min(FMA peak, AI x HBM peak), AI =
    algorithmic flops / algorithmic bytes."""
    info = model.info()
    calls = sum(i["n_residual_evals"] for i in infos)
    ms = sum(i["ms_residual"] for i in infos)
    if calls == 0 or ms <= 0.0 or not fma_gflops:
        return None
    per_s = (ms / calls) / 1000.0
    flops, nbytes = float(info["residual_flops"]), float(info["residual_bytes"])
    hbm, hbm_kind = hbm_peak()
    ai = flops / nbytes
    attainable = min(fma_gflops, ai * hbm)
    achieved = flops / per_s / 1e9
    return {"kernel": "residual", "bound": "fma" if fma_gflops <= ai * hbm else "hbm",
            "achieved": achieved, "unit": "GFLOP/s", "fma_peak": fma_gflops,
            "fma_peak_source": f"measured live ({fma_kind} FMA microbenchmark, efem_fma_peak)",
            "hbm_peak_source": hbm_kind, "arithmetic_intensity": ai, "attainable": attainable,
            "frac": achieved / attainable, "mean_launch_us": per_s * 1e6}


def roofline_report(model, infos):
    """Return (roofline dict, mean kernel launches per solve)."""
    info = model.info()
    n3 = model.n_dof
    res_calls = sum(i["n_residual_evals"] for i in infos)
    res_ms = sum(i["ms_residual"] for i in infos)
    pc_calls = sum(i["n_precond_applies"] for i in infos)
    pc_ms = sum(i["ms_precond"] for i in infos)
    tot_ms = sum(i["ms_total"] for i in infos)
    fac_ms = sum(i["ms_factor"] for i in infos)
    res_bytes = float(info["residual_bytes"])
    pc_bytes = 2.0 * 8.0 * info["factor_nnz"] + 5.0 * 8.0 * n3
    groups = {
        "residual": (res_ms, res_calls, res_bytes),
        "precond_apply": (pc_ms, pc_calls, pc_bytes),
    }
    dom = max(groups, key=lambda k: groups[k][0])
    ms, calls, nbytes = groups[dom]
    per_launch_s = (ms / max(calls, 1)) / 1000.0
    achieved = nbytes / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
    peak, kind = hbm_peak()
    roof = {
        "kernel": dom,
        "bound": "hbm",
        "achieved": achieved,
        "peak": peak,
        "peak_source": kind,
        "unit": "GB/s",
        "frac": achieved / peak,
        "traffic": measured_traffic(dom),
        "algorithmic_bytes_per_launch": nbytes,
        "launches_timed": calls,
        "mean_launch_us": per_launch_s * 1e6,
        "share_of_solve": {"residual": res_ms / tot_ms, "precond_apply": pc_ms / tot_ms,
                           "factorisation": fac_ms / tot_ms,
                           "other (line search, two-loop, host waits)": max(0.0, 1.0 - (res_ms + pc_ms + fac_ms) / tot_ms)},
    }
    if dom == "residual":
        roof["residual_gflops_fp64"] = info["residual_flops"] / per_launch_s / 1e9
    launches = sum(i["n_kernel_launches"] for i in infos) / len(infos)
    return roof, launches
