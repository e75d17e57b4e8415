"""Runs of the named benchmark configurations, printed as JSON lines.

  python -m euler3d_b200.report c1    # 64x32x2 bump channel, Mach 0.5, CFL 1.5, 2000 RK5 iterations
  python -m euler3d_b200.report c2    # 256x128x4 biconvex O-grid (262,144 prisms), Mach 0.8, AoA 1.25,
                                      # CFL 1.2, Roe and AUSM: FP64 and FP32_FLUX toward a 1e-8
                                      # density-residual drop (at most 200,000 iterations), the
                                      # residual drop at checkpoints, the FP32 fields and lift / drag
                                      # against FP64 after the same iterations, and where the FP32
                                      # residual stalls
  python -m euler3d_b200.report c5    # the served stream at its stated sizes (10k-2M cells), FP64
                                      # and ladder served against the plain path, per tolerance
  python -m euler3d_b200.report c4    # 256 uneven instances (bump channels and biconvex O-grids of
                                      # 5k-200k cells, Mach 0.3-0.85, AoA -4..6, Roe/AUSM) run as
                                      # one batch to a 1e-8 drop, FP32_FLUX then FP64, against the
                                      # plain one-at-a-time FP64 path on a sample of them

Meshes are generated in-process (synthetic, seeded).  The FP64 solution stands for the oracle at
this size: the FP64 path equals the CPU restatement to 1e-10 per cell on the small cases the tests
run (running the CPU restatement to convergence on 262k cells takes hours).
"""
from __future__ import annotations

import json
import sys
import time

import numpy as np

from . import _lib
from . import meshgen as mg
from . import serve
from .solver import EulerSolver, FlowConfig, Mesh


def _fields_error(a, b, n):
    speed = np.sqrt(b["u"][:n] ** 2 + b["v"][:n] ** 2 + b["w"][:n] ** 2)
    out = {}
    for k in ("rho", "u", "v", "w", "p", "E"):
        scale = speed if k in ("u", "v", "w") else np.abs(b[k][:n])
        out[k] = float(np.max(np.abs(a[k][:n] - b[k][:n]) / scale))
    return out


def c1():
    arrays = Mesh.from_raw(mg.bump_channel(64, 32, 2)).arrays()
    out = []
    for prec, name in ((_lib.PREC_FP64, "fp64"), (_lib.PREC_FP32_FLUX, "fp32")):
        s = EulerSolver(arrays, FlowConfig(mach=0.5, aoa=0.0, cfl=1.5, precision=prec, ordering=_lib.ORDER_SPATIAL))
        st = s.run(2000, sampling=2000)
        out.append({"config": "c1", "precision": name, "cells": int(arrays["n_cells"]), "iterations": st["iterations"],
                    "device_ms": st["device_ms"], "ms_per_iteration": st["device_ms"] / st["iterations"],
                    "last_rms": st["last_rms"], "rms0": float(s.rms_history()[0]), "cl": st["cl"], "cd": st["cd"]})
    return out


def c2(max_iter=200_000):
    t = time.time()
    arrays = Mesh.from_raw(mg.biconvex_ogrid(256, 128, 4)).arrays()
    prep_s = time.time() - t
    n = int(arrays["n_cells"])
    out = []
    checkpoints = [1000, 10_000, 50_000, 100_000, 150_000, max_iter]
    # CL / CD as the reference selects them (MESH_ORIENTATION: force y and force x, not rotated)
    cl = lambda f: float(f[1])  # noqa: E731
    cd = lambda f: float(f[0])  # noqa: E731
    for scheme, sname in ((_lib.SCHEME_ROE, "roe"), (_lib.SCHEME_AUSM, "ausm")):
        flow = dict(mach=0.8, aoa=1.25, cfl=1.2, scheme=scheme, ordering=_lib.ORDER_SPATIAL)
        row = {"config": "c2", "scheme": sname, "cells": n, "mesh_prep_s": prep_s}
        res = {}
        for prec, name in ((_lib.PREC_FP64, "fp64"), (_lib.PREC_FP32_FLUX, "fp32")):
            s = EulerSolver(arrays, FlowConfig(precision=prec, **flow))
            st = s.run(max_iter, sampling=1_000_000, min_residual_drop=1e-8, check_every=256)
            f, _ = s.coefficients()
            h = s.rms_history()
            res[name] = (s.get_state(), f)
            row[name] = {"iterations": st["iterations"], "stop": st["stop_reason"], "device_s": st["device_ms"] / 1e3,
                         "drop_at": {str(k): float(h[min(k, h.size) - 1] / h[0]) for k in checkpoints},
                         "best_drop": float(h.min() / h[0]), "cl": cl(f), "cd": cd(f)}
        (g64, f64), (g32, f32) = res["fp64"], res["fp32"]
        row["fp32_vs_fp64_same_iterations"] = {
            "fields_max_rel": _fields_error(g32, g64, n),
            "cl_rel": abs(cl(f32) - cl(f64)) / max(abs(cl(f64)), 1e-12),
            "cd_rel": abs(cd(f32) - cd(f64)) / max(abs(cd(f64)), 1e-12)}
        # where the FP32 residual stalls (the ladder's switch point)
        s = EulerSolver(arrays, FlowConfig(precision=_lib.PREC_FP32_FLUX, **flow))
        st = s.run(max_iter, sampling=1_000_000, stall_window=2000, stall_below=1e-2, check_every=256)
        h = s.rms_history()
        row["fp32_stall"] = {"iterations": st["iterations"], "stop": st["stop_reason"], "drop": float(h.min() / h[0])}
        out.append(row)
    return out


def c4(n=256, max_iter=20_000, plain_sample=32):
    """n instances drawn with seed 3 (bump channels and biconvex O-grids, cells log-uniform in
    [5k, 200k], Mach uniform in [0.3, 0.85], AoA in [-4, 6] degrees, Roe or AUSM), all present at
    the start, each to a 1e-8 density-residual drop (at most max_iter iterations).  They run as one
    batch with the precision ladder: FP32_FLUX until a solve's residual stalls, then FP64 from that
    state.  Beside it the plain FP64 path solves the first plain_sample instances one at a time;
    its solves/s on that sample stands for the whole set (solving all of them one at a time would
    take several minutes more), and its lift and drag are compared with the batch's.  Wall-clock
    spans include the host mesh preparation (four threads) in both."""
    reqs = serve.request_stream(n, 0.0, cells=(5000, 200_000), seed=3, drops=(1e-8,),
                                schemes=(_lib.SCHEME_ROE, _lib.SCHEME_AUSM))
    srv = serve.Server(max_members=n, ladder=True, max_iter=max_iter)
    served = srv.serve(reqs)
    row = {"config": "c4", "instances": n, "cells_total": int(sum(r.cells for r in served)), "max_iter": max_iter,
           "batch_ladder": serve.summarize(served), "peak_members": srv.peak_members,
           "peak_device_bytes": srv.peak_bytes, "device_busy_s": srv.step_ms / 1e3,
           "fp32_iteration_share": (sum(r.fp32_iterations for r in served) /
                                    max(sum(max(r.iterations, 0) for r in served), 1))}
    b = row["batch_ladder"]
    b["cell_stage_updates_per_s"] = 5.0 * b["cell_iterations"] / b["seconds"]
    sample = [q for q in reqs if q.rid < plain_sample]
    base = serve.serve_plain(sample, max_iter=max_iter)
    p = serve.summarize(base)
    p["cell_stage_updates_per_s"] = 5.0 * p["cell_iterations"] / p["seconds"]
    row["plain_sample"] = p
    row["plain_sample_size"] = len(sample)
    d = serve._diffs(base, [r for r in served if r.rid < plain_sample])
    row["sample_diffs"] = {k: d[k] for k in ("max_rel_diff_cl", "max_rel_diff_cd", "converged_max_rel_diff_cl",
                                             "converged_max_rel_diff_cd", "same_outcome")}
    row["speedup_solves_per_s"] = b["solves_per_s"] / p["solves_per_s"]
    # converged solves only: the rate of solves that reached the 1e-8 drop, batch against plain
    row["speedup_converged_solves_per_s"] = (b["converged_solves_per_s"] / p["converged_solves_per_s"]
                                             if p["converged"] else None)
    return [row]


def c5(n=64, rate=20.0, max_iter=20_000):
    """The served request stream at its stated size distribution: n requests (Poisson arrivals at
    `rate` per second, seed 4), meshes of 10k-2M cells log-uniform (bump channels and biconvex
    O-grids; O-grid requests above 1M cells get a channel, see serve.request_mesh), Mach 0.3-0.85,
    AoA -4..6, Roe or AUSM, tolerance 1e-6 or 1e-8, admission by device-memory footprint under a
    150 GB budget.  Served in FP64 and with the FP32 -> FP64 precision ladder, then solved one at a
    time by the plain FP64 path; solves/s, p50/p99 latency, and converged solves/s for each
    tolerance apart.  The stated stream runs 600 s (12,000 requests); this is its first n."""
    reqs = serve.request_stream(n, rate, cells=(10_000, 2_000_000), seed=4, drops=(1e-6, 1e-8),
                                schemes=(_lib.SCHEME_ROE, _lib.SCHEME_AUSM))
    out = serve.compare(reqs, _lib.PREC_FP64, max_iter=max_iter, ladder=True, hbm_budget=150e9)
    out["config"] = "c5"
    out["workload"] = (f"{n} requests, Poisson {rate:g}/s (seed 4), cells log-uniform [10000, 2000000], "
                       f"Mach 0.3-0.85, AoA -4..6, Roe/AUSM, drop 1e-6/1e-8, max_iter {max_iter}, 150 GB budget")
    out["cells_total"] = int(sum(q.cells for q in reqs))
    for key in ("served", "served_ladder"):
        if key in out and "plain" in out:
            out[key]["speedup_converged_solves_per_s"] = (
                out[key]["converged_solves_per_s"] / out["plain"]["converged_solves_per_s"]
                if out["plain"]["converged"] else None)
    return [out]


def main(argv=None):
    which = (argv or sys.argv[1:] or ["c1"])[0]
    rows = {"c1": c1, "c2": c2, "c4": c4, "c5": c5}[which]()
    for r in rows:
        print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
