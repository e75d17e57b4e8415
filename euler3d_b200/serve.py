"""Served solves: a continuous-batching request loop on one device.

Requests (a mesh from the synthetic generators, Mach, angle of attack, residual-drop tolerance)
arrive over time.  Each is prepared on host threads (mesh generation, connectivity, metrics),
admitted when its device-memory footprint fits the budget, created on the device and added to the
running :class:`~euler3d_b200.batch.Batch`, where it shares every launch with the solves already
running; it is retired -- and its memory freed -- as soon as its own stop test fires.  State stays
on the device from admission to retirement.

:func:`serve_plain` runs the same request stream the plain way, one solve at a time with
:meth:`EulerSolver.run` in FP64, for comparison.  No counterpart in the reference, which runs one
solve per process.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import dataclasses
import math
import threading
import time
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import _lib
from . import meshgen as mg
from .batch import Batch
from .solver import EulerSolver, FlowConfig, Mesh


@dataclasses.dataclass
class SolveRequest:
    rid: int
    arrival: float            # seconds after the stream starts
    family: str               # "channel" (bump channel, hexahedra) or "ogrid" (biconvex O-grid, prisms; channel above 600k cells)
    cells: int                # requested size; the generated mesh has about this many cells
    mach: float
    aoa: float                # degrees
    drop: float               # the solve ends when the density RMS falls below drop x its first RMS
    scheme: int = _lib.SCHEME_ROE
    seed: int = 0


@dataclasses.dataclass
class SolveResult:
    rid: int
    cells: int
    arrival: float
    admitted: float           # added to the batch (served) or started (plain)
    finished: float
    iterations: int
    stop_reason: int
    status: int
    cl: float
    cd: float
    cm: float
    last_rms: float
    device_bytes: int
    fp32_iterations: int = 0  # ladder: iterations of the FP32_FLUX phase
    drop: float = 0.0         # the request's residual-drop tolerance

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def request_stream(n: int, rate: float, cells: Sequence[int] = (10_000, 2_000_000), seed: int = 4,
                   drops: Sequence[float] = (1e-6, 1e-8), mach: Sequence[float] = (0.3, 0.85),
                   aoa: Sequence[float] = (-4.0, 6.0), families: Sequence[str] = ("channel", "ogrid"),
                   schemes: Sequence[int] = (_lib.SCHEME_ROE,)) -> List[SolveRequest]:
    """``n`` requests with Poisson arrivals at ``rate`` per second (``rate`` <= 0: all at time 0),
    log-uniform cell counts, uniform Mach and angle of attack, drawn from one seeded generator."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, n) if rate > 0 else np.zeros(n)
    arrivals = np.cumsum(gaps) - (gaps[0] if n else 0.0)
    lo, hi = math.log(cells[0]), math.log(cells[1])
    out = []
    for i in range(n):
        out.append(SolveRequest(
            rid=i, arrival=float(arrivals[i]), family=str(families[int(rng.integers(len(families)))]),
            cells=int(round(math.exp(rng.uniform(lo, hi)))), mach=float(rng.uniform(*mach)),
            aoa=float(rng.uniform(*aoa)), drop=float(drops[int(rng.integers(len(drops)))]),
            scheme=int(schemes[int(rng.integers(len(schemes)))]), seed=int(rng.integers(1 << 30))))
    return out


def request_mesh(req: SolveRequest) -> mg.RawMesh:
    """The generator mesh of a request, sized to about ``req.cells``: a bump channel of nx = 2 ny
    hexahedra x 2 layers, or a biconvex O-grid of 2 nj x nj hexahedra x 2 span layers split into
    prisms.  The O-grid's radial stretch is scaled so that its total growth is that of 128 layers
    at 1.1, and its span layers are 0.1 chord thick, thinner on grids finer than 128 radial layers:
    the reference's tetrahedron volume (from edge lengths, src/mesh/Metrics.cpp:311-331) loses a
    flat cell's volume to cancellation when its span edges are long against its in-plane ones,
    which happens first at the sharp leading and trailing edges of a fine grid.  Above about 800k
    cells the O-grid's slivers still lose their volume that way (measured: the smallest such grid
    of a sweep over 200k-1M cells had 815,863 cells), so requests above 600k cells get a channel."""
    if req.family == "ogrid" and req.cells <= 600_000:
        nj = max(4, int(round(math.sqrt(req.cells / 8.0))))
        dz = 0.1 * min(1.0, 128.0 / nj)
        return mg.biconvex_ogrid(2 * nj, nj, 2, seed=req.seed % 1000, stretch=1.1 ** (128.0 / nj), span=2 * dz)
    if req.family in ("channel", "ogrid"):
        ny = max(4, int(round(math.sqrt(req.cells / 4.0))))
        return mg.bump_channel(2 * ny, ny, 2, seed=req.seed % 1000)
    raise ValueError(f"unknown mesh family {req.family!r}")


def request_flow(req: SolveRequest, precision: int) -> FlowConfig:
    cfl = 1.5 if req.family == "channel" else 1.2
    return FlowConfig(mach=req.mach, aoa=req.aoa, cfl=cfl, scheme=req.scheme, precision=precision,
                      ordering=_lib.ORDER_SPATIAL)


def footprint_estimate(n_cells: int, n_faces: int, precision: int) -> int:
    """Upper estimate of a solver's device memory (e3d_solver_info.device_bytes) from its mesh
    size: per cell the two state buffers, W0, E, Mach, geometry, CSR and tile lists; per face its
    geometry, gather entries and tile records (counted twice for faces shared by two tiles)."""
    per_cell = 96 + 40 + 8 + 8 + 32 + 4 + 8 + 12 + 16
    per_face = 32 + 16 + 2 * 40 + 8 + 64
    if precision == _lib.PREC_FP32_FLUX:
        per_cell += 2 * 32 + 16
        per_face += 2 * 24
    return int(1.25 * (per_cell * n_cells + per_face * n_faces)) + (1 << 20)


def final_coefficients(solver: EulerSolver):
    """(CL, CD, CM) of the solver's current state: AeroCoefficients::Update
    (src/solver/AeroCoefficients.cpp:38-52) with the flow's MESH_ORIENTATION axes and signs."""
    f, m = solver.coefficients()
    fl = solver.flow
    return (float(f[fl.cl[0]] * fl.cl[1]), float(f[fl.cd[0]] * fl.cd[1]), float(m[fl.cm[0]] * fl.cm[1]))


def _prepare(req: SolveRequest) -> dict:
    return Mesh.from_raw(request_mesh(req)).arrays()


def percentile(xs: Sequence[float], q: float) -> float:
    return float(np.percentile(np.asarray(xs, dtype=float), q)) if len(xs) else float("nan")


def summarize(results: Sequence[SolveResult], t_end: Optional[float] = None) -> Dict[str, float]:
    """Solves/s over the stream's span (first arrival to last completion), latency percentiles, and how
    the solves ended: converged (residual-drop test), capped (max_iter) or diverged (non-finite)."""
    if not results:
        return {"solves": 0}
    t0 = min(r.arrival for r in results)
    t1 = t_end if t_end is not None else max(r.finished for r in results)
    lat = [r.latency for r in results]
    span = max(t1 - t0, 1e-9)
    def conv(r):
        return r.status == _lib.E3D_OK and r.stop_reason == _lib.STOP_RESIDUAL

    converged = sum(conv(r) for r in results)
    # the solves of each tolerance apart: how many reached it, at what rate, with what latency
    by_drop = {}
    for d in sorted({r.drop for r in results}):
        rs = [r for r in results if r.drop == d]
        ok = [r for r in rs if conv(r)]
        by_drop[f"{d:g}"] = {"requests": len(rs), "converged": len(ok), "converged_solves_per_s": len(ok) / span,
                             "p50_latency_s": percentile([r.latency for r in rs], 50),
                             "p99_latency_s": percentile([r.latency for r in rs], 99),
                             "converged_p50_latency_s": percentile([r.latency for r in ok], 50)}
    return {"solves": len(results), "seconds": t1 - t0, "solves_per_s": len(results) / span, "by_drop": by_drop,
            "refused": sum(r.status not in (_lib.E3D_OK, _lib.E3D_ERR_NONFINITE, _lib.E3D_ERR_TIMEOUT) for r in results),
            "converged": converged, "converged_solves_per_s": converged / span,
            "capped": sum(r.status == _lib.E3D_OK and r.stop_reason == _lib.STOP_MAX_ITER for r in results),
            "diverged": sum(r.status == _lib.E3D_ERR_NONFINITE for r in results),
            "p50_latency_s": percentile(lat, 50), "p99_latency_s": percentile(lat, 99),
            "mean_latency_s": float(np.mean(lat)),
            "cell_iterations": float(sum(r.cells * max(r.iterations, 0) for r in results))}


class Server:
    """Continuous batching of solve requests on one device.

    ``hbm_budget`` bounds the summed device memory of the admitted solves (an estimate reserved at
    admission, replaced by the handle's own figure once it exists); ``max_members`` bounds how many
    run at once; ``iterations_per_step`` is the graph length between admissions and retirements.

    With ``ladder`` every solve runs first in FP32_FLUX (fluxes in single precision, about 1.7x the
    FP64 throughput) until its tolerance or until its residual has set no new minimum for
    ``stall_window`` iterations once it is below ``stall_below`` x its first value -- the floor
    single-precision fluxes put under the residual; initial transients do not count -- and
    then continues in FP64 from that state to the same absolute residual the plain FP64 solve stops
    at (the tolerance times the solve's first RMS).  The result is the FP64 solution."""

    def __init__(self, device: int = 0, precision: int = _lib.PREC_FP64, hbm_budget: float = 150e9,
                 max_members: int = 256, iterations_per_step: int = 32, max_iter: int = 200_000,
                 prep_workers: int = 4, sampling: int = 1_000_000, ladder: bool = False, stall_window: int = 200,
                 stall_below: float = 1e-2,
                 clock: Callable[[], float] = time.perf_counter):
        self.device, self.precision = device, precision
        self.budget, self.max_members = float(hbm_budget), max_members
        self.every, self.max_iter, self.sampling = iterations_per_step, max_iter, sampling
        self.prep_workers, self.clock = prep_workers, clock
        self.ladder, self.stall_window, self.stall_below = ladder, stall_window, stall_below
        self.peak_bytes = 0
        self.peak_members = 0
        self.steps = 0
        self.step_ms = 0.0

    def serve(self, requests: Sequence[SolveRequest], on_result: Optional[Callable] = None) -> List[SolveResult]:
        first = _lib.PREC_FP32_FLUX if self.ladder else self.precision
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        prep = cf.ThreadPoolExecutor(self.prep_workers, thread_name_prefix="e3d-prep")
        device_pool = cf.ThreadPoolExecutor(1, thread_name_prefix="e3d-device")  # creation and release
        preparing = collections.deque()   # (req, future -> arrays)
        ready = collections.deque()       # (req, arrays, estimate)
        creating = collections.deque()    # dicts: req, fut -> solver, est, phase, ...
        members: Dict[int, dict] = {}     # id(solver) -> dict: req, solver, admitted, bytes, phase, ...
        results: List[SolveResult] = []
        used = 0.0
        batches = [Batch(self.device)] + ([Batch(self.device)] if self.ladder else [])
        steppers = cf.ThreadPoolExecutor(len(batches), thread_name_prefix="e3d-step")  # batches run concurrently
        t0 = self.clock()
        wake = threading.Event()

        def create(req, arrays, prec, state=None):
            s = EulerSolver(arrays, request_flow(req, prec), autotune=False)
            if state is not None:
                s.set_state(state)
            wake.set()
            return s

        def finish(m, s, st, status, iterations, fp32_iterations):
            req = m["req"]
            cl, cd, cm = final_coefficients(s)
            r = SolveResult(req.rid, s.n_cells, req.arrival, m["admitted"], self.clock() - t0, iterations,
                            st["stop_reason"], status, cl, cd, cm, st["last_rms"], m["bytes"], fp32_iterations,
                            drop=req.drop)
            results.append(r)
            if on_result:
                on_result(r, s)

        try:
            while pending or preparing or ready or creating or members:
                now = self.clock() - t0
                while pending and pending[0].arrival <= now:
                    req = pending.popleft()
                    fut = prep.submit(_prepare, req)
                    fut.add_done_callback(lambda _f: wake.set())
                    preparing.append((req, fut))
                while preparing and preparing[0][1].done():
                    req, fut = preparing.popleft()
                    try:
                        arrays = fut.result()
                    except _lib.E3DError as e:  # a mesh the preparation refuses: a failed request
                        results.append(SolveResult(req.rid, req.cells, req.arrival, math.nan, self.clock() - t0, 0,
                                                   -1, e.status, math.nan, math.nan, math.nan, math.nan, 0,
                                                   drop=req.drop))
                        continue
                    est = footprint_estimate(int(arrays["n_cells"]), int(arrays["n_faces"]), first)
                    ready.append((req, arrays, est))
                # admission by device-memory footprint, first come first served
                while ready and len(members) + len(creating) < self.max_members:
                    req, arrays, est = ready[0]
                    if est > self.budget:  # can never fit: refused, not queued for ever
                        ready.popleft()
                        results.append(SolveResult(req.rid, int(arrays["n_cells"]), req.arrival, math.nan,
                                                   self.clock() - t0, 0, -1, _lib.E3D_ERR_OOM, math.nan, math.nan,
                                                   math.nan, math.nan, est, drop=req.drop))
                        continue
                    if used + est > self.budget:
                        break
                    ready.popleft()
                    used += est
                    creating.append({"req": req, "fut": device_pool.submit(create, req, arrays, first), "est": est,
                                     "phase": 1, "arrays": arrays if self.ladder else None,
                                     "admitted": self.clock() - t0})
                while creating and creating[0]["fut"].done():
                    c = creating.popleft()
                    s = c["fut"].result()
                    nbytes = int(s.info()["device_bytes"])
                    used += nbytes - c["est"]
                    m = dict(c, solver=s, bytes=nbytes)
                    del m["fut"]
                    req = c["req"]
                    if c["phase"] == 1:
                        m["admitted"] = self.clock() - t0
                        batches[0].add(s, max_iter=self.max_iter, sampling=self.sampling, min_residual_drop=req.drop,
                                       stall_window=self.stall_window if self.ladder else 0,
                                       stall_below=self.stall_below)
                    else:
                        batches[1].add(s, max_iter=max(self.max_iter - c["it1"], 0), sampling=self.sampling,
                                       min_residual=c["rms0"] * req.drop)
                    members[id(s)] = m
                self.peak_bytes = max(self.peak_bytes, used)
                self.peak_members = max(self.peak_members, len(members))
                if members:
                    # each batch on its own stream: the ladder's two batches overlap on the device
                    running = [b for b in batches if b.info()["n_running"]]
                    for f in [steppers.submit(b.step, self.every) for b in running]:
                        f.result()
                    for b in running:
                        self.steps += 1
                        self.step_ms += b.info()["last_step_ms"]
                    for phase, b in enumerate(batches, start=1):
                        for s, st, status in b.retire():
                            m = members.pop(id(s))
                            if (phase == 1 and self.ladder and status == _lib.E3D_OK
                                    and st["stop_reason"] == _lib.STOP_STALL):
                                # FP32 floor reached: continue in FP64 from this state
                                rms0 = float(s.rms_history()[0])
                                state = s.get_state()
                                est = footprint_estimate(s.n_cells, int(m["arrays"]["n_faces"]), _lib.PREC_FP64)
                                used += est
                                creating.append({"req": m["req"], "est": est, "phase": 2, "it1": st["iterations"],
                                                 "rms0": rms0, "admitted": m["admitted"], "arrays": None,
                                                 "fut": device_pool.submit(create, m["req"], m["arrays"],
                                                                           _lib.PREC_FP64, state)})
                            elif phase == 1:
                                finish(m, s, st, status, st["iterations"], st["iterations"] if self.ladder else 0)
                            else:
                                finish(m, s, st, status, m["it1"] + st["iterations"], m["it1"])
                            used -= m["bytes"]
                            device_pool.submit(s.close)
                else:
                    # idle: wait for the next arrival, a finished preparation or a created solver
                    wake.clear()
                    timeout = (pending[0].arrival - now) if pending else 0.05
                    if not (preparing and preparing[0][1].done()) and not (creating and creating[0]["fut"].done()):
                        wake.wait(max(0.0, min(timeout, 0.05)))
        finally:
            steppers.shutdown(wait=True)
            for b in batches:
                b.close()
            prep.shutdown(wait=True)
            device_pool.shutdown(wait=True)
        return results


def serve_plain(requests: Sequence[SolveRequest], device: int = 0, precision: int = _lib.PREC_FP64,
                max_iter: int = 200_000, prep_workers: int = 4, sampling: int = 1_000_000,
                clock: Callable[[], float] = time.perf_counter,
                on_result: Optional[Callable] = None) -> List[SolveResult]:
    """The plain path on the same stream: meshes prepared on the same host threads as they arrive,
    solves run one at a time in arrival order with :meth:`EulerSolver.run` (autotuned stage kernel)."""
    reqs = sorted(requests, key=lambda r: r.arrival)
    prep = cf.ThreadPoolExecutor(prep_workers, thread_name_prefix="e3d-prep")
    results: List[SolveResult] = []
    t0 = clock()
    futures = []
    timers = []
    try:
        for req in reqs:  # each preparation starts when its request arrives
            f: cf.Future = cf.Future()
            futures.append(f)

            def start(req=req, f=f):
                try:
                    f.set_result(_prepare(req))
                except BaseException as e:  # noqa: BLE001 - handed to the consumer
                    f.set_exception(e)

            t = threading.Timer(max(0.0, req.arrival - (clock() - t0)), lambda st=start: prep.submit(st))
            t.start()
            timers.append(t)
        for req, f in zip(reqs, futures):
            try:
                arrays = f.result()
            except _lib.E3DError as e:  # a mesh the preparation refuses: a failed request
                now = clock() - t0
                results.append(SolveResult(req.rid, req.cells, req.arrival, now, now, 0, -1, e.status, math.nan,
                                           math.nan, math.nan, math.nan, 0, drop=req.drop))
                continue
            started = clock() - t0
            s = EulerSolver(arrays, request_flow(req, precision))
            status = _lib.E3D_OK
            try:
                st = s.run(max_iter, sampling=sampling, min_residual_drop=req.drop)
            except _lib.E3DError as e:
                status, st = e.status, getattr(e, "stats", {"iterations": -1, "stop_reason": -1, "last_rms": math.nan})
            finished = clock() - t0
            cl, cd, cm = final_coefficients(s)
            r = SolveResult(req.rid, s.n_cells, req.arrival, started, finished, st["iterations"],
                            st["stop_reason"], status, cl, cd, cm, st["last_rms"], int(s.info()["device_bytes"]),
                            drop=req.drop)
            results.append(r)
            if on_result:
                on_result(r, s)
            s.close()
    finally:
        for t in timers:
            t.cancel()
        prep.shutdown(wait=True)
    return results


def _diffs(base: Sequence[SolveResult], other: Sequence[SolveResult]) -> Dict[str, object]:
    """Lift and drag differences between two runs of the same requests: over every solve that ended
    without error in both, and over those that reached their tolerance in both (a solve stopped at
    max_iter is unconverged, and two paths to the same iteration count need not agree there)."""
    by = {r.rid: r for r in other}
    ok = [b for b in base if b.status == _lib.E3D_OK and by[b.rid].status == _lib.E3D_OK]
    conv = [b for b in ok if b.stop_reason == _lib.STOP_RESIDUAL and by[b.rid].stop_reason == _lib.STOP_RESIDUAL]

    # relative to the coefficient's size, at least 1e-2 (a near-zero lift has no relative error)
    def rel(rs, key):
        d = [abs(getattr(b, key) - getattr(by[b.rid], key)) / max(abs(getattr(b, key)), 1e-2) for b in rs]
        return max(d) if d else None

    mism = [b for b in base if (b.status, b.stop_reason) != (by[b.rid].status, by[b.rid].stop_reason)]
    return {"max_rel_diff_cl": rel(ok, "cl"), "max_rel_diff_cd": rel(ok, "cd"),
            "converged_max_rel_diff_cl": rel(conv, "cl"), "converged_max_rel_diff_cd": rel(conv, "cd"),
            "same_outcome": not mism,
            "outcome_mismatches": [{"rid": b.rid, "cells": b.cells, "plain": [b.status, b.stop_reason, b.iterations],
                                    "served": [by[b.rid].status, by[b.rid].stop_reason, by[b.rid].iterations]}
                                   for b in mism]}


def compare(requests: Sequence[SolveRequest], precision: int = _lib.PREC_FP64, iterations_per_step: int = 32,
            hbm_budget: float = 150e9, max_members: int = 256, prep_workers: int = 4,
            plain: bool = True, max_iter: int = 200_000, ladder: bool = False) -> Dict[str, object]:
    """Serve ``requests`` with continuous batching (in ``precision``, and with ``ladder`` also with the
    FP32 -> FP64 precision ladder), then (``plain``) the same stream one solve at a time in FP64;
    solves/s, latency percentiles, and the largest lift / drag difference from the plain solves."""
    srv = Server(precision=precision, iterations_per_step=iterations_per_step, hbm_budget=hbm_budget,
                 max_members=max_members, prep_workers=prep_workers, max_iter=max_iter)
    served = srv.serve(requests)
    out: Dict[str, object] = {"requests": len(requests), "served": summarize(served),
                              "served_precision": {0: "fp64_exact", 1: "fp64", 2: "fp32"}[precision],
                              "peak_members": srv.peak_members, "peak_device_bytes": srv.peak_bytes,
                              "device_busy_s": srv.step_ms / 1e3,
                              "failed": sum(r.status != _lib.E3D_OK for r in served)}
    lad = None
    if ladder:
        ls = Server(iterations_per_step=iterations_per_step, hbm_budget=hbm_budget, max_members=max_members,
                    prep_workers=prep_workers, max_iter=max_iter, ladder=True)
        lad = ls.serve(requests)
        out["served_ladder"] = summarize(lad)
        out["served_ladder"]["fp32_iteration_share"] = (sum(r.fp32_iterations for r in lad) /
                                                        max(sum(max(r.iterations, 0) for r in lad), 1))
        out["served_ladder"]["device_busy_s"] = ls.step_ms / 1e3
    if plain:
        base = serve_plain(requests, prep_workers=prep_workers, max_iter=max_iter)
        out["plain"] = summarize(base)
        out.update(_diffs(base, served))
        out["max_iteration_diff"] = max(abs(b.iterations - r.iterations) for b, r in
                                        zip(sorted(base, key=lambda r: r.rid), sorted(served, key=lambda r: r.rid)))
        out["speedup_solves_per_s"] = out["served"]["solves_per_s"] / out["plain"]["solves_per_s"]
        if lad is not None:
            d = _diffs(base, lad)
            out["served_ladder"].update({k: d[k] for k in ("max_rel_diff_cl", "max_rel_diff_cd", "converged_max_rel_diff_cl",
                                                           "converged_max_rel_diff_cd", "same_outcome")})
            out["served_ladder"]["speedup_solves_per_s"] = (out["served_ladder"]["solves_per_s"] /
                                                            out["plain"]["solves_per_s"])
    return out


def main(argv: Optional[Sequence[str]] = None) -> None:
    import argparse
    import json

    ap = argparse.ArgumentParser(description="Serve a synthetic request stream; compare with one-at-a-time solves.")
    ap.add_argument("--requests", type=int, default=32)
    ap.add_argument("--rate", type=float, default=20.0, help="Poisson arrivals per second (0: all at once)")
    ap.add_argument("--cells", type=int, nargs=2, default=(10_000, 200_000))
    ap.add_argument("--drops", type=float, nargs="+", default=(1e-6, 1e-8))
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--every", type=int, default=32)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--detail", action="store_true", help="print one line per served request")
    ap.add_argument("--max-iter", type=int, default=200_000)
    ap.add_argument("--ladder", action="store_true", help="also serve with the FP32 -> FP64 precision ladder")
    a = ap.parse_args(argv)
    reqs = request_stream(a.requests, a.rate, cells=a.cells, seed=a.seed, drops=a.drops,
                          schemes=(_lib.SCHEME_ROE, _lib.SCHEME_AUSM))
    prec = {"fp64": _lib.PREC_FP64, "fp32": _lib.PREC_FP32_FLUX}[a.precision]
    if a.detail:
        srv = Server(precision=prec, iterations_per_step=a.every, hbm_budget=a.budget_gb * 1e9, max_iter=a.max_iter)
        for r in sorted(srv.serve(reqs), key=lambda r: r.rid):
            q = reqs[r.rid]
            print(json.dumps({"rid": r.rid, "family": q.family, "cells": r.cells, "mach": round(q.mach, 3),
                              "aoa": round(q.aoa, 2), "scheme": q.scheme, "drop": q.drop, "iterations": r.iterations,
                              "stop": r.stop_reason, "status": r.status, "cl": r.cl, "cd": r.cd,
                              "latency_s": round(r.latency, 3), "last_rms": r.last_rms}), flush=True)
        return
    print(json.dumps(compare(reqs, prec, a.every, a.budget_gb * 1e9, plain=not a.no_plain, max_iter=a.max_iter,
                             ladder=a.ladder)), flush=True)


if __name__ == "__main__":
    main()
