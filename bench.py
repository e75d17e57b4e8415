#!/usr/bin/env python
"""Benchmark of the Euler3D explicit-solver hot path on B200: RK-stage cell-updates/s.

Workload (default): the large all-tetrahedral roofline mesh -- a 128^3 hexahedral box [0,4]^3
with a Gaussian floor bump (height 0.1, sigma 0.3), every hexahedron split into 6 tetrahedra
(12,582,912 cells, 25,264,128 faces), nodes jittered 3% (seed 2), Mach 0.6, AoA 0, Roe, CFL 1.0,
FP64, Morton (spatial) cell order on the device.  Synthetic, generated in-process (no dataset).

A step is one RK5 iteration (5 stages over every cell, with ghost updates, local time step,
update, density-RMS reduction and force sampling).  ``value`` counts 5 x cells x steps per
second with the state resident in HBM; ``e2e`` is the same metric through the C ABI with host
buffers: the flow state is copied in from pinned host memory and read back every call.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): independent replicas, no data-path collective; the
timing is the max over ranks.  ``--impl reference`` times the reference's own CPU solver program
(compiled from its sources with its Release flags into oracle/_ref/fast) on the same mesh through
its multi-rank MPI path, one rank per host core, or the CPU oracle port if that binary is absent.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK-stage cell-updates/s"
# SAMPLING= of the timed runs in both arms: the force coefficients (AeroCoefficients::Update) are
# sampled at the first iteration of a run only, as the reference arm's config sets it, so the metric
# counts the RK stages and the per-iteration RMS, not force sampling.
SAMPLING = 1_000_000_000
UNIT = "cell-updates/s"
WORKLOAD = "bump_box_tets 128^3x6 (12,582,912 tets), Mach 0.6, Roe, RK5, CFL 1.0"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=128, help="hexahedra per box edge (6 tets each)")
    ap.add_argument("--precision", choices=["fp64", "fp64_exact", "fp32"], default="fp64")
    ap.add_argument("--ordering", choices=["spatial", "rcm", "native"], default="spatial")
    ap.add_argument("--kernel", type=int, default=0,
                    help="stage kernel: 0 autotuned, 1/2 gather, 3 face tiles, 4 warp-specialised persistent face tiles, "
                         "5 face tiles at 7 blocks/SM (FP32_FLUX: 8 blocks/SM)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--mode", choices=["all", "stage", "served", "profile", "kernels"], default="all",
                    help="stage: the RK-stage line only; served: the served-stream comparison only; profile: a "
                         "few iterations of one stage-kernel variant (--kernel, no autotuning) on the --n mesh, "
                         "for profiler captures of a small case; kernels: a few launches of every other kernel "
                         "(residual smoothing, state transfers, batch stage / RMS / coefficients / control) on "
                         "small cases, for profiler captures")
    ap.add_argument("--batch-kernel", choices=["tiles", "ws"], default="tiles",
                    help="kernels mode: the batch stage kernel (one block per tile, or warp-specialised)")
    ap.add_argument("--iters", type=int, default=2, help="profile mode: RK5 iterations")
    ap.add_argument("--channel", type=int, nargs=2, default=None, metavar=("NX", "NY"),
                    help="profile mode: a 2-layer bump channel of NX x NY x 2 hexahedra instead of the tetrahedral box")
    ap.add_argument("--ref-mesh", choices=["c3", "c1", "c2"], default="c3",
                    help="reference arm: the bench mesh (c3), the 64x32x2 bump channel of config 1 (Mach 0.5, "
                         "CFL 1.5) or the 256x128x4 biconvex O-grid of config 2 (Mach 0.8, AoA 1.25, CFL 1.2)")
    ap.add_argument("--ref-ranks", type=int, default=0, help="reference arm: MPI ranks (0: one per host core)")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the check of the first iteration against the CPU oracle")
    ap.add_argument("--served-requests", type=int, default=48)
    ap.add_argument("--served-rate", type=float, default=20.0, help="Poisson arrivals per second (0: burst)")
    ap.add_argument("--served-cells", type=int, nargs=2, default=(5_000, 50_000))
    ap.add_argument("--served-max-iter", type=int, default=20_000)
    return ap.parse_args()


def served_leg(args) -> dict:
    """The served-stream comparison: a seeded Poisson stream of solve requests (bump-channel and
    biconvex O-grid meshes, log-uniform cell counts, Mach 0.3-0.85, AoA -4..6 deg, Roe or AUSM,
    residual-drop tolerance 1e-6 or 1e-8, at most ``served_max_iter`` iterations each) served with
    continuous batching in FP64 and with the FP32 -> FP64 precision ladder, then the same stream solved
    one at a time (plain FP64 path)."""
    from euler3d_b200 import _lib, serve

    lo, hi = args.served_cells
    reqs = serve.request_stream(args.served_requests, args.served_rate, cells=(lo, hi), seed=4,
                                drops=(1e-6, 1e-8), schemes=(_lib.SCHEME_ROE, _lib.SCHEME_AUSM))
    out = serve.compare(reqs, _lib.PREC_FP64, max_iter=args.served_max_iter, ladder=True)
    out["workload"] = (f"{args.served_requests} requests, Poisson {args.served_rate:g}/s (seed 4), "
                       f"cells log-uniform [{lo}, {hi}], Mach 0.3-0.85, AoA -4..6, Roe/AUSM, drop 1e-6/1e-8, "
                       f"max_iter {args.served_max_iter}")
    out["metric"] = "served solves/s, p50/p99 latency"
    return out


def batch_leg(device: int, peak: float) -> dict:
    """Batched members (configuration 4's shape): 64 bump channels of about 20k and of about 80k
    cells (Mach 0.30-0.615, CFL 1.5, Roe) advanced together, FP64 and FP32_FLUX, 20 RK5 iterations
    timed after 4 untimed; cell-stage updates per second over the members, and the stage kernel's
    roofline fraction from the algorithmic bytes of the members' meshes (the graph's device time
    includes the per-iteration RMS / coefficient kernels, so the fraction is a lower bound)."""
    from euler3d_b200 import _lib, meshgen
    from euler3d_b200.batch import Batch
    from euler3d_b200.solver import EulerSolver, FlowConfig, Mesh

    out = {}
    for nx, ny in ((140, 70), (280, 140)):
        arrays = Mesh.from_raw(meshgen.bump_channel(nx, ny, 2)).arrays()
        n, f = int(arrays["n_cells"]), int(arrays["n_faces"])
        for prec, name in ((_lib.PREC_FP64, "fp64"), (_lib.PREC_FP32_FLUX, "fp32")):
            members = [EulerSolver(arrays, FlowConfig(mach=0.3 + 0.005 * i, cfl=1.5, precision=prec,
                                                      ordering=_lib.ORDER_SPATIAL, device=device), autotune=False)
                       for i in range(64)]
            b = Batch(device)
            for m in members:
                b.add(m, 100)
            b.step(4)
            b.step(20)
            ms = b.info()["last_step_ms"]
            b.close()
            for m in members:
                m.close()
            rate = 5.0 * 20 * 64 * n / (ms / 1e3)
            bpc = algorithmic_bytes_per_cell_stage(n, f, fp32=prec == _lib.PREC_FP32_FLUX)
            out[f"{n}_cells_{name}"] = {"members": 64, "cells_per_member": n, "faces_per_cell": f / n,
                                        "step_ms_20_iterations": ms, "cell_stage_updates_per_s": rate,
                                        "bytes_per_cell_stage": bpc, "achieved_GBs": rate * bpc / 1e9,
                                        "frac_of_measured_peak": rate * bpc / 1e9 / peak}
    return out


def algorithmic_bytes_per_cell_stage(n_cells: int, n_faces: int, fp32: bool = False) -> float:
    """Bytes per cell-stage, each array counted once with ideal gather reuse (f_c = faces per cell).
    FP64: 160 + 40 f_c -- read W, read U0, write W (3 x 40 B), 1/5 of writing U0 (8 B), volume
    (8 B), sum|S| (24 B); per face 2 x int32 + (nx, ny, nz, S) x 8 B.
    FP32 flux / FP64 state: 104 + 24 f_c -- 5 x 4 B primitives read and written, U0 read in double,
    float volume and sum|S|; per face 2 x int32 + 4 x 4 B."""
    fc = n_faces / n_cells
    return (104.0 + 24.0 * fc) if fp32 else (160.0 + 40.0 * fc)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(key: str = "dram_bytes_per_cell"):
    """DRAM bytes per cell and stage-kernel launch from the committed ncu summary (scaled to this mesh
    by the caller): as captured (``dram_bytes_per_cell``), or the reads plus the new states' writes
    that must reach DRAM over many launches (``dram_bytes_per_cell_steady``)."""
    path = os.path.join(ROOT, "profiles", "stage_kernel_tets.txt")
    try:
        vals = {}
        for line in open(path):
            if "=" in line and not line.startswith("#"):
                k, v = line.split("=", 1)
                vals[k.strip()] = v.strip()
        return float(vals[key])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms while the timed region runs (a power
    cap moves the SM clock on that time scale)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.06)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                f_sm, f_max = float(parts[1]), float(parts[2])
            except ValueError:
                continue
            sm.append(f_sm)
            smax.append(f_max)
            try:
                power.append(float(parts[3]))
            except ValueError:
                pass
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_min_mhz": min(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "power_w_max": max(power) if power else None,
                "reasons": sorted(reasons), "samples": len(sm)}


class Replicas:
    """The bookkeeping of a run on N GPUs, one process each.  Each rank solves its own whole copy of
    the workload (replicas: the solver path has no data-path exchange), so the only collectives are
    the barriers around the timed region and the max over ranks of its duration; the job's rate is
    the units every rank processed over the slowest rank's time.  ``dist`` is torch.distributed
    (or None for one process); ``device`` holds the reduction's tensor ("cuda:i" with NCCL, "cpu"
    with gloo)."""

    def __init__(self, dist, device: str):
        self.dist, self.device = dist, device

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        if self.dist is None:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    @staticmethod
    def rate(units_per_rank: float, world: int, seconds: float) -> float:
        """Whole-job throughput: ``units_per_rank`` on each of ``world`` ranks in ``seconds`` (the
        max over ranks)."""
        return units_per_rank * world / seconds


# --------------------------------------------------------------------------------------- ours
def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch

    from euler3d_b200 import _lib, meshgen
    from euler3d_b200.solver import STATE_KEYS, EulerSolver, FlowConfig, Mesh

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    if args.mode == "served":
        if rank == 0:
            print(json.dumps({"metric": "served solves/s", "n_gpus": 1, "served": served_leg(args)}), flush=True)
        return
    if args.mode == "profile":
        profile_case(args, local_rank)
        return
    if args.mode == "kernels":
        kernels_case(args, local_rank)
        return

    t0 = time.time()
    raw = meshgen.bump_box_tets(args.n)
    arrays = Mesh.from_raw(raw).arrays()
    del raw
    n_cells, n_faces = int(arrays["n_cells"]), int(arrays["n_faces"])
    prec = {"fp64": _lib.PREC_FP64, "fp64_exact": _lib.PREC_FP64_EXACT, "fp32": _lib.PREC_FP32_FLUX}[args.precision]
    order = {"spatial": _lib.ORDER_SPATIAL, "rcm": _lib.ORDER_RCM, "native": _lib.ORDER_NATIVE}[args.ordering]
    flow = FlowConfig(mach=0.6, aoa=0.0, cfl=1.0, precision=prec, ordering=order, device=local_rank)
    stream = torch.cuda.Stream(device=local_rank)
    solver = EulerSolver(arrays, flow, stream=stream.cuda_stream)
    setup_s = time.time() - t0
    K, W = args.steps, args.warmup

    replicas = Replicas(dist, f"cuda:{local_rank}")
    barrier, max_over_ranks = replicas.barrier, replicas.max

    # warm-up: same graph chunk as the timed run (the graph is instantiated here, not while timing)
    solver.run(W, check_every=K, stage_kernel=args.kernel, sampling=SAMPLING)

    # ---- timed region: state resident in HBM
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ev0.record(stream)
    stats = solver.run(K, check_every=K, sampling=SAMPLING)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    assert stats["iterations"] == K, stats
    value = Replicas.rate(5.0 * n_cells * K, world, ms / 1e3)

    # ---- stage-kernel duration for the roofline: the timed region's K-iteration graph run once
    # more, right after it, with an event pair captured around every stage kernel (on the solver's
    # stream), so the stages run back to back under the same sustained load.  The event nodes slow
    # a graph by a few percent, which is why the timed region itself carries none.  For context
    # also the launches timed alone (direct launches, the host waiting after every iteration).
    tstats = solver.run(K, check_every=K, profile_stages=2, sampling=SAMPLING)
    stage_ms = tstats["stage_ms"] / tstats["stage_launches"]
    prof = solver.run(max(K // 5, 4), profile_stages=1, sampling=SAMPLING)
    stage_ms_alone = prof["stage_ms"] / prof["stage_launches"]
    bytes_per_cell = algorithmic_bytes_per_cell_stage(n_cells, n_faces, fp32=args.precision == "fp32")
    achieved = bytes_per_cell * n_cells / (stage_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    tr = profiled_traffic() if args.precision != "fp32" else None
    tr_steady = profiled_traffic("dram_bytes_per_cell_steady") if args.precision != "fp32" else None

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        T = solver.state_size
        host_in = {k: torch.empty(T, dtype=torch.float64).pin_memory().numpy() for k in STATE_KEYS}
        host_out = {k: torch.empty(T, dtype=torch.float64).pin_memory().numpy() for k in STATE_KEYS}
        solver.set_freestream()
        solver.get_state(host_in)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        solver.set_state(host_in)
        st2 = solver.run(K, check_every=K, sampling=SAMPLING)
        solver.get_state(host_out)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ems = max_over_ranks(e0.elapsed_time(e1))
        assert st2["iterations"] == K
        nbytes = 8 * T * 8
        e2e = {"value": Replicas.rate(5.0 * n_cells * K, world, ems / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": nbytes / K, "d2h_bytes_per_step": nbytes / K,
               "ms": ems, "note": "set_state (pinned host -> device) + run(K) + get_state (device -> pinned host)"}

    # ---- CPU baseline: the oracle port, one RK5 iteration of the same mesh, one core; and parity of
    # the GPU's first iteration from the freestream with that iteration (outside every timed region)
    cpu, parity = None, None
    if rank == 0 and world == 1 and not (args.no_cpu_baseline and args.no_parity):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po  # the checker and the CPU baseline only

        m = po.Mesh(arrays)
        fl = po.flow(0.6, 0.0, 1.4, 1.0)
        s = po.freestream(m, fl)
        t = time.time()
        po.run(m, fl, s, 1)
        dt = time.time() - t
        if not args.no_cpu_baseline:
            cpu = {"value": 5.0 * n_cells / dt, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"1 RK5 iteration of the full {n_cells}-cell mesh ({dt:.1f} s), CPU oracle port, 1 thread"}
        if not args.no_parity:
            parity = first_iteration_parity(solver, arrays, flow, s.a, n_cells, args.precision)

    launches = stats["kernel_launches"]
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 flux / f64 state" if args.precision == "fp32" else "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cells": n_cells, "faces": n_faces, "faces_per_cell": n_faces / n_cells,
                   "precision": args.precision, "ordering": args.ordering,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (state + mesh ~3 GB per replica)", "setup_s": round(setup_s, 1),
                   "sampling": SAMPLING},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": (tr * n_cells if tr else None),
                     "traffic_steady": (tr_steady * n_cells if tr_steady else None),
                     "traffic_note": "ncu capture of one launch on the 1.57M-tet box, per cell, scaled to this mesh; "
                                     "traffic_steady adds the new states' writes still in L2 when the captured "
                                     "launch ended (written back later)",
                     "peak_kind": peak_kind,
                     "kernel": (["-", "-", "tile_kernel_f32<4>", "tile_ws_kernel<WS_F32>", "tile_kernel_f32<8>", "-", "-"]
                                if args.precision == "fp32" else
                                ["stage_kernel<false,4>", "stage_kernel<false,5>", "tile_kernel<false,4>",
                                 "tile_ws_kernel<WS_FAST>", "tile_kernel<false,7>", "colour_kernel<128> (per class)",
                                 "colour_kernel<512> (per class)"])[solver.info()["stage_variant"]],
                     "bytes_per_cell_stage": bytes_per_cell,
                     "avg_launch_ms": stage_ms, "launches_timed": tstats["stage_launches"],
                     "timing": "event pairs around every stage kernel in a second run of the timed graph",
                     "frac_alone": bytes_per_cell * n_cells / (stage_ms_alone / 1e3) / 1e9 / peak,
                     "avg_launch_ms_alone": stage_ms_alone, "autotune": solver.info()},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk, "parity": parity,
    }
    solver.close()

    def extra(fn, *a):
        # the legs after the headline measurement: a failure in one is reported in its own key and
        # does not cost the line
        try:
            return fn(*a)
        except Exception as exc:  # noqa: BLE001
            print(f"bench: {fn.__name__} failed: {exc!r}", file=sys.stderr, flush=True)
            return {"error": repr(exc)[:300]}

    if rank == 0 and world == 1 and args.mode == "all" and args.precision == "fp64":
        line["fp32_flux"] = extra(fp32_flux_leg, arrays, flow, n_cells, n_faces, K, W, peak, local_rank)
    del arrays
    if rank == 0 and world == 1 and args.mode == "all":
        line["batch"] = extra(batch_leg, local_rank, peak)
    if rank == 0 and world == 1 and args.mode == "all" and args.served_requests > 0:
        line["served"] = extra(served_leg, args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def fp32_flux_leg(arrays, flow, n_cells: int, n_faces: int, K: int, W: int, peak: float, device: int) -> dict:
    """The FP32_FLUX mode (fluxes, face states and time step in single precision; state, RK
    accumulation and reductions in double) on the bench mesh: K RK5 iterations timed with CUDA events
    after W untimed, the stage kernel's roofline fraction from its algorithmic bytes (104 + 24 f_c per
    cell-stage), and its error against the FP64 path after the same W + K iterations from the
    freestream (interior fields, velocity relative to the local speed; the wall force vector)."""
    import dataclasses

    import numpy as np
    import torch

    from euler3d_b200 import _lib
    from euler3d_b200.solver import EulerSolver

    stream = torch.cuda.Stream(device=device)
    s32 = EulerSolver(arrays, dataclasses.replace(flow, precision=_lib.PREC_FP32_FLUX), stream=stream.cuda_stream)
    s32.run(W, check_every=K, sampling=SAMPLING)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    st = s32.run(K, check_every=K, sampling=SAMPLING)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    assert st["iterations"] == K, st
    g32, f32 = s32.get_state(), s32.coefficients()[0]
    prof = s32.run(K, check_every=K, profile_stages=2, sampling=SAMPLING)
    stage_ms = prof["stage_ms"] / prof["stage_launches"]
    variant = s32.info()["stage_variant"]
    s32.close()
    s64 = EulerSolver(arrays, dataclasses.replace(flow, precision=_lib.PREC_FP64), autotune=False)
    s64.run(W + K, check_every=K, sampling=SAMPLING)
    g64, f64 = s64.get_state(), s64.coefficients()[0]
    s64.close()
    speed = np.sqrt(g64["u"][:n_cells] ** 2 + g64["v"][:n_cells] ** 2 + g64["w"][:n_cells] ** 2)
    err = {}
    for k in ("rho", "u", "v", "w", "p", "E", "H"):
        scale = speed if k in ("u", "v", "w") else np.abs(g64[k][:n_cells])
        err[k] = float(np.max(np.abs(g32[k][:n_cells] - g64[k][:n_cells]) / scale))
    bpc = algorithmic_bytes_per_cell_stage(n_cells, n_faces, fp32=True)
    return {"value": 5.0 * n_cells * K / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / K, "steps": K, "warmup": W,
            "stage_kernel": ["-", "-", "tile_kernel_f32<4>", "tile_ws_kernel<WS_F32>", "tile_kernel_f32<8>", "-", "-"][variant],
            "avg_launch_ms": stage_ms, "bytes_per_cell_stage": bpc,
            "achieved_GBs": bpc * n_cells / (stage_ms / 1e3) / 1e9,
            "frac": bpc * n_cells / (stage_ms / 1e3) / 1e9 / peak,
            "vs_fp64": {"iterations": W + K, "start": "freestream", "fields_max_rel": err,
                        "force_rel": float(np.linalg.norm(np.subtract(f32, f64)) / max(np.linalg.norm(f64), 1e-300))}}


def first_iteration_parity(solver, arrays, flow, oracle_state, n_cells, precision):
    """One RK5 iteration of the benchmarked mesh from the freestream on the GPU against the same
    iteration of the CPU oracle: the largest per-cell relative difference of the interior fields
    (velocity components relative to the local flow speed), and, for the double-precision modes, a
    bit-for-bit check of FP64_EXACT on the same mesh."""
    import dataclasses

    import numpy as np

    from euler3d_b200 import _lib
    from euler3d_b200.solver import EulerSolver

    def max_rel(g, o):
        speed = np.sqrt(o["u"][:n_cells] ** 2 + o["v"][:n_cells] ** 2 + o["w"][:n_cells] ** 2)
        worst = 0.0
        for k in ("rho", "u", "v", "w", "p", "E", "H"):
            scale = speed if k in ("u", "v", "w") else np.abs(o[k][:n_cells])
            worst = max(worst, float(np.max(np.abs(g[k][:n_cells] - o[k][:n_cells]) / scale)))
        return worst

    solver.set_freestream()
    solver.run(1)
    out = {"cells": n_cells, "iterations": 1, "start": "freestream", "against": "CPU oracle (C restatement)",
           "max_rel": max_rel(solver.get_state(), oracle_state),
           "tolerance": 2e-5 if precision == "fp32" else 1e-10}
    out["within_tolerance"] = out["max_rel"] <= out["tolerance"]
    if precision != "fp32":
        ex = EulerSolver(arrays, dataclasses.replace(flow, precision=_lib.PREC_FP64_EXACT), autotune=False)
        ex.run(1)
        g = ex.get_state()
        ex.close()
        out["fp64_exact_bitwise"] = bool(all(np.array_equal(g[k][:n_cells], oracle_state[k][:n_cells])
                                             for k in ("rho", "u", "v", "w", "p", "E", "H")))
    return out


def profile_case(args, device):
    """A few RK5 iterations of one stage-kernel variant on the --n bump box (autotuning skipped when a
    kernel is forced, so the only stage launches are the run's), for profiler captures of a small
    case; prints the cell count and the mean stage-kernel duration (CUDA events)."""
    from euler3d_b200 import _lib, meshgen
    from euler3d_b200.solver import EulerSolver, FlowConfig, Mesh

    prec = {"fp64": _lib.PREC_FP64, "fp64_exact": _lib.PREC_FP64_EXACT, "fp32": _lib.PREC_FP32_FLUX}[args.precision]
    order = {"spatial": _lib.ORDER_SPATIAL, "rcm": _lib.ORDER_RCM, "native": _lib.ORDER_NATIVE}[args.ordering]
    if args.channel:
        arrays = Mesh.from_raw(meshgen.bump_channel(args.channel[0], args.channel[1], 2)).arrays()
        flow = FlowConfig(mach=0.5, cfl=1.5, precision=prec, ordering=order, device=device)
    else:
        arrays = Mesh.from_raw(meshgen.bump_box_tets(args.n)).arrays()
        flow = FlowConfig(mach=0.6, cfl=1.0, precision=prec, ordering=order, device=device)
    s = EulerSolver(arrays, flow, autotune=args.kernel == 0)
    st = s.run(args.iters, profile_stages=True, stage_kernel=args.kernel)
    print(json.dumps({"mode": "profile", "cells": int(arrays["n_cells"]), "kernel": args.kernel,
                      "precision": args.precision, "autotune_ms": s.info()["variant_ms"],
                      "stage_ms": st["stage_ms"] / st["stage_launches"]}), flush=True)


def kernels_case(args, device):
    """A few launches of each kernel that is not a solo stage kernel, on small cases, for profiler
    captures: explicit Euler with residual smoothing on the --n bump box (residual phase, two
    smoothing passes, update), the state loaders and readers (FP64 and FP32_FLUX), and a batch of 64
    bump channels of 19,600 cells in FP64 and in FP32_FLUX (batch stage, RMS, coefficient and
    control-gather kernels; --batch-kernel chooses the FP64 stage kernel).  Prints the device time of
    each part, and the batch stage throughput."""
    from euler3d_b200 import _lib, meshgen
    from euler3d_b200.batch import Batch
    from euler3d_b200.solver import EulerSolver, FlowConfig, Mesh

    out = {"mode": "kernels"}
    arrays = Mesh.from_raw(meshgen.bump_box_tets(args.n)).arrays()
    out["cells"] = int(arrays["n_cells"])
    sm = EulerSolver(arrays, FlowConfig(mach=0.6, cfl=1.0, precision=_lib.PREC_FP64, ordering=_lib.ORDER_SPATIAL,
                                        integrator=_lib.INTEGRATOR_EULER, smoothing=True, device=device),
                     autotune=False)
    out["smoothing_ms"] = sm.run(args.iters)["device_ms"]
    sm.set_state(sm.get_state())
    sm.close()
    f32 = EulerSolver(arrays, FlowConfig(mach=0.6, cfl=1.0, precision=_lib.PREC_FP32_FLUX,
                                         ordering=_lib.ORDER_SPATIAL, device=device), autotune=False)
    f32.set_state(f32.get_state())
    f32.close()
    ch = Mesh.from_raw(meshgen.bump_channel(140, 70, 2)).arrays()
    for prec, name in ((_lib.PREC_FP64, "fp64"), (_lib.PREC_FP32_FLUX, "fp32")):
        b = Batch(device)
        if prec == _lib.PREC_FP64 and args.batch_kernel == "ws":
            b.set_kernel(_lib.BATCH_KERNEL_WS)
        members = [EulerSolver(ch, FlowConfig(mach=0.3 + 0.005 * i, cfl=1.5, precision=prec, ordering=_lib.ORDER_SPATIAL,
                                              device=device), autotune=False) for i in range(64)]
        for m in members:
            b.add(m, 4 * args.iters)
        b.step(args.iters)
        b.step(args.iters)
        ms = b.info()["last_step_ms"]
        it = args.iters + (args.iters & 1)
        out[f"batch_{name}_step_ms"] = ms
        out[f"batch_{name}_cell_stages_per_s"] = 5.0 * it * 64 * int(ch["n_cells"]) / (ms / 1e3)
        b.close()
        for m in members:
            m.close()
    print(json.dumps(out), flush=True)


# --------------------------------------------------------------------------------------- reference
REF_MPI = os.path.join(ROOT, "oracle", "_ref", "fast", "e3d_ref_mpi")


def host_cores() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def run_reference_mpi(raw, arrays, ranks: int, warm: int, iters: int, mach: float, cfl: float, workdir: str,
                      aoa: float = 0.0) -> dict:
    """The reference's own solver program on ``ranks`` host cores through its multi-rank path:
    the mesh cut into ``ranks`` x-slab partitions (.par files in the reference's layout), each rank
    one process (shared-memory MPI), EulerSolver::Run timed by the driver over ``iters`` iterations
    after ``warm`` untimed ones.  Built with the reference's Release flags (-Ofast)."""
    from euler3d_b200 import meshgen

    pattern = os.path.join(workdir, "part_#.par")
    meshgen.write_partitions(raw, ranks, pattern, arrays=arrays)
    cfg = meshgen.CaseConfig(mach=mach, aoa=aoa, cfl=cfl, max_iter=iters, sampling=SAMPLING)
    cfg_path = os.path.join(workdir, "case.e3d")
    meshgen.write_e3d(cfg, cfg_path, pattern, os.path.join(workdir, "out.dat"), n_partitions=ranks)
    env = dict(os.environ, E3D_MPI_RANKS=str(ranks))
    r = subprocess.run([REF_MPI, cfg_path, str(warm), str(iters), "fast"], capture_output=True, text=True, env=env,
                       cwd=workdir, start_new_session=True, timeout=3600)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("E3D_REF_MPI ")]
    if r.returncode != 0 or not lines:
        raise RuntimeError(f"reference run failed (rc {r.returncode}): {r.stderr[-400:]}")
    return json.loads(lines[-1][len("E3D_REF_MPI "):])


def run_reference(args, rank, world):
    """``--impl reference``: the reference's own CPU solver on the bench's workload, on this host's
    cores.  Under torchrun only rank 0 runs it."""
    if rank != 0:
        return
    from euler3d_b200 import meshgen
    from euler3d_b200.solver import Mesh

    K, W = args.steps, max(args.warmup, 3)
    cores = host_cores()
    aoa = 0.0
    if args.ref_mesh == "c1":
        raw, mach, cfl = meshgen.bump_channel(64, 32, 2), 0.5, 1.5
        workload = "bump_channel 64x32x2 (4,096 hexahedra), Mach 0.5, Roe, RK5, CFL 1.5"
    elif args.ref_mesh == "c2":
        raw, mach, cfl, aoa = meshgen.biconvex_ogrid(256, 128, 4), 0.8, 1.2, 1.25
        workload = "biconvex O-grid 256x128x4 (262,144 prisms), Mach 0.8, AoA 1.25, Roe, RK5, CFL 1.2"
    else:
        raw, mach, cfl = meshgen.bump_box_tets(args.n), 0.6, 1.0
        workload = WORKLOAD
    cells = raw.n_cells
    if os.path.exists(REF_MPI):
        ranks = args.ref_ranks if args.ref_ranks > 0 else max(1, min(cores, 64))
        arrays = Mesh.from_raw(raw).arrays()
        with tempfile.TemporaryDirectory(prefix="e3dref") as d:
            res = run_reference_mpi(raw, arrays, ranks, W, K, mach, cfl, d, aoa=aoa)
        assert res["cells"] == cells and res["iterations"] == K, res
        tmax = res["seconds"]
        value = 5.0 * cells * K / tmax
        kind = "reference"
        sample = (f"the reference's solver program (EulerSolver::Run, compiled from the reference sources with its "
                  f"Release flags -Ofast) on the full {cells}-cell mesh, {ranks} MPI ranks (one process per host core, "
                  f"x-slab partitions, the reference's halo exchange over a shared-memory MPI), {K} timed RK5 "
                  f"iterations after {W} untimed; slowest rank {tmax:.2f} s; mesh connectivity set up by the "
                  f"library's numbering-identical preparation ({res['setup_seconds']:.1f} s setup)")
        config = {"workload": workload, "cells": cells, "ranks": ranks, "host_cores": cores,
                  "build": "-Ofast (reference Release)", "same_mesh": args.ref_mesh == "c3", "sampling": SAMPLING}
    else:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po  # the CPU baseline only

        arrays = Mesh.from_raw(raw).arrays()
        m = po.Mesh(arrays)
        fl = po.flow(mach, aoa, 1.4, cfl)
        s = po.freestream(m, fl)
        po.run(m, fl, s, 1)
        t = time.time()
        po.run(m, fl, s, 1)
        tmax = (time.time() - t) * K
        ranks = 1
        value = 5.0 * cells / (tmax / K)
        kind = "port"
        sample = (f"CPU oracle port (the reference binary is not built), 1 RK5 iteration of the full {cells}-cell "
                  f"mesh, 1 thread, scaled to {K} steps")
        config = {"workload": workload, "cells": cells, "ranks": 1, "same_mesh": args.ref_mesh == "c3"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": tmax * 1e3 / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference", "config": config,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ranks, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
