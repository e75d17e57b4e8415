"""Runs of the named benchmark configurations, printed as JSON lines.

  python -m euler3d_b200.report c1    # 64x32x2 bump channel, Mach 0.5, CFL 1.5, 2000 RK5 iterations
  python -m euler3d_b200.report c2    # 256x128x4 biconvex O-grid (262,144 prisms), Mach 0.8, AoA 1.25,
                                      # CFL 1.2, Roe and AUSM: FP64 and FP32_FLUX toward a 1e-8
                                      # density-residual drop (at most 200,000 iterations), the
                                      # residual drop at checkpoints, the FP32 fields and lift / drag
                                      # against FP64 after the same iterations, and where the FP32
                                      # residual stalls

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


def main(argv=None):
    which = (argv or sys.argv[1:] or ["c1"])[0]
    rows = {"c1": c1, "c2": c2}[which]()
    for r in rows:
        print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
