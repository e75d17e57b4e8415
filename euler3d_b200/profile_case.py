"""Run a few RK5 iterations of one stage-kernel variant on a bump-box tetrahedral mesh, for profiling.

  python -m euler3d_b200.profile_case --n 64 --kernel 5 --precision fp64 --iters 2

Prints the cell count, the autotuner's timings and the mean stage-kernel duration (CUDA events).
With a forced ``--kernel`` the autotuner is skipped, so the only stage launches are the run's.
"""
import argparse

from . import _lib, meshgen
from .solver import EulerSolver, FlowConfig, Mesh


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64, help="hexahedra per box edge (6 tetrahedra each)")
    ap.add_argument("--kernel", type=int, default=0, help="0 autotuned, 1/2 gather, 3 face tiles, 4 pipelined tiles, "
                                                               "5 face tiles at 7 blocks/SM")
    ap.add_argument("--precision", choices=["fp64", "fp64_exact", "fp32"], default="fp64")
    ap.add_argument("--iters", type=int, default=2)
    args = ap.parse_args()
    prec = {"fp64": _lib.PREC_FP64, "fp64_exact": _lib.PREC_FP64_EXACT, "fp32": _lib.PREC_FP32_FLUX}[args.precision]
    arrays = Mesh.from_raw(meshgen.bump_box_tets(args.n)).arrays()
    s = EulerSolver(arrays, FlowConfig(mach=0.6, cfl=1.0, precision=prec, ordering=_lib.ORDER_SPATIAL),
                    autotune=args.kernel == 0)
    info = s.info()
    st = s.run(args.iters, profile_stages=True, stage_kernel=args.kernel)
    print(f"cells {arrays['n_cells']} autotune {info['variant_ms']} chosen {info['stage_variant']} "
          f"stage_ms {st['stage_ms'] / st['stage_launches']:.4f}")


if __name__ == "__main__":
    main()
