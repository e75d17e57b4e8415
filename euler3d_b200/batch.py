"""Many solvers advanced together in shared launches (``e3d_batch_*`` of include/euler3d_b200.h).

Each Runge-Kutta stage of every running member is one kernel over the members' concatenated face
tiles; the RMS / stop tests and the force coefficients are one block per member of two more
kernels; a step's iterations are one CUDA graph.  A member computes exactly what
``EulerSolver.run(..., stage_kernel=KERNEL_TILE)`` computes for it alone.  No counterpart in the
reference, which solves one mesh per process.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Tuple

from . import _lib
from ._lib import check
from .solver import EulerSolver, run_params, stats_dict


class Batch:
    def __init__(self, device: int = 0, stream: Optional[int] = None):
        h = C.c_void_p()
        check(_lib.load().e3d_batch_create(device, stream, C.byref(h)))
        self._h = h
        self._members: Dict[int, EulerSolver] = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.load().e3d_batch_destroy(self._h)
            self._h = None
            self._members.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_kernel(self, kernel: int) -> None:
        """``e3d_batch_set_kernel``: BATCH_KERNEL_TILES (one block per member tile) or BATCH_KERNEL_WS
        (the warp-specialised persistent kernel; FP64 modes)."""
        check(_lib.load().e3d_batch_set_kernel(self._h, kernel))

    def __len__(self) -> int:
        return len(self._members)

    def add(self, solver: EulerSolver, max_iter: int, sampling: int = 1, min_residual: float = 0.0,
            min_aerocoeff_error: float = 0.0, min_residual_drop: float = 0.0, stall_window: int = 0,
            stall_below: float = 0.0) -> None:
        """Start a run of ``solver`` in the batch (stop criteria as in :meth:`EulerSolver.run`)."""
        rp = run_params(max_iter, sampling, min_residual, min_aerocoeff_error, min_residual_drop=min_residual_drop,
                        stall_window=stall_window, stall_below=stall_below)
        check(_lib.load().e3d_batch_add(self._h, solver._h, C.byref(rp)))
        self._members[solver._h.value] = solver

    def step(self, iterations: int = 32) -> int:
        """Run ``iterations`` (rounded up to even) more iterations of every running member; returns
        the number of members still running."""
        n = C.c_int32()
        check(_lib.load().e3d_batch_step(self._h, iterations, C.byref(n)))
        return n.value

    def retire(self) -> List[Tuple[EulerSolver, Dict[str, object], int]]:
        """Members whose runs have stopped, taken out of the batch: (solver, stats, status)."""
        cap = max(len(self._members), 1)
        hs = (C.c_void_p * cap)()
        sts = (_lib.RunStats * cap)()
        status = (C.c_int * cap)()
        n = C.c_int32()
        check(_lib.load().e3d_batch_retire(self._h, hs, sts, status, cap, C.byref(n)))
        out = []
        for i in range(n.value):
            solver = self._members.pop(hs[i])
            out.append((solver, stats_dict(sts[i]), int(status[i])))
        return out

    def remove(self, solver: EulerSolver) -> Dict[str, object]:
        st = _lib.RunStats()
        check(_lib.load().e3d_batch_remove(self._h, solver._h, C.byref(st)))
        self._members.pop(solver._h.value, None)
        return stats_dict(st)

    def run_all(self, iterations_per_step: int = 32):
        """Step until no member runs; returns (solver, stats, status) of every member in retirement order."""
        done = []
        while self._members:
            self.step(iterations_per_step)
            done.extend(self.retire())
        return done

    def info(self) -> Dict[str, object]:
        i = _lib.BatchInfo()
        check(_lib.load().e3d_batch_info_get(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in _lib.BatchInfo._fields_}
