"""The reference's multi-rank CPU path, as the CPU baseline runs it (oracle/_ref/fast/e3d_ref_mpi:
the unmodified reference sources with the reference's Release flags, over the shared-memory MPI of
oracle/ref/mpi_shm).  Test infrastructure: these check the baseline, not the product.

* The fast connectivity the timing driver uses on large meshes (the library's numbering-identical
  mesh preparation in place of the reference's O(N^2) searches) changes nothing: a 4-rank run gives
  every rank's flow state bit for bit as the reference's own connectivity does.
* The shared-memory MPI carries the reference's halo exchange and collectives correctly: 4 ranks
  agree with 1 rank on the same mesh to the level at which the reference's discretisation depends
  on cell numbering (the entropy fix's left cell, partition-interface ghosts), far below what a
  missing or misplaced halo value would cause.
"""
import os
import subprocess

import numpy as np
import pytest

from euler3d_b200 import meshgen as mg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_MPI = os.path.join(ROOT, "oracle", "_ref", "fast", "e3d_ref_mpi")
pytestmark = pytest.mark.skipif(not os.path.exists(REF_MPI), reason="reference timing build missing (make -C oracle ref-fast)")


def run(tmp, raw, ranks, iters, fast, tag):
    d = tmp / tag
    d.mkdir()
    pattern = str(d / "part_#.par")
    mg.write_partitions(raw, ranks, pattern)
    cfg = mg.CaseConfig(mach=0.5, cfl=1.5, max_iter=iters, sampling=1_000_000)
    mg.write_e3d(cfg, str(d / "case.e3d"), pattern, str(d / "out.dat"), n_partitions=ranks)
    env = dict(os.environ, E3D_MPI_RANKS=str(ranks), E3D_REF_DUMP=str(d), E3D_MPI_TIMEOUT="120")
    r = subprocess.run([REF_MPI, str(d / "case.e3d"), "0", str(iters)] + (["fast"] if fast else []), cwd=d,
                       env=env, capture_output=True, text=True, timeout=300, start_new_session=True)
    assert r.returncode == 0, r.stderr[-2000:]
    assert any(ln.startswith("E3D_REF_MPI ") for ln in r.stdout.splitlines())
    return [np.fromfile(d / f"state_{k}.f64").reshape(8, -1) for k in range(ranks)]


def test_fast_connectivity_is_the_references(tmp_path):
    raw = mg.bump_channel(32, 16, 2)
    slow = run(tmp_path, raw, 4, 12, False, "slow")
    fast = run(tmp_path, raw, 4, 12, True, "fast")
    for a, b in zip(slow, fast):
        assert np.array_equal(a, b)


def test_ranks_agree_with_one_rank(tmp_path):
    raw = mg.bump_channel(32, 16, 2)
    one = run(tmp_path, raw, 1, 12, True, "one")[0]
    four = run(tmp_path, raw, 4, 12, True, "four")
    # each part's elements are the global elements of its slab in ascending order (write_partitions)
    n = raw.n_cells
    cx = raw.xyz[raw.elem_nodes, 0].mean(axis=1)
    part = np.empty(n, np.int64)
    part[np.argsort(cx, kind="stable")] = np.arange(n) * 4 // n
    merged = np.empty((8, n))
    for p in range(4):
        cells = np.flatnonzero(part == p)
        merged[:, cells] = four[p][:, : cells.size]
    ref = one[:, :n]
    for k in (0, 4, 5):  # rho, p, E
        rel = np.max(np.abs(merged[k] - ref[k]) / np.abs(ref[k]))
        assert rel < 1e-5, (k, rel)  # measured 1e-7..5e-7 after 12 iterations


@pytest.mark.parametrize("mesh,extra", [("c3", ["--n", "8"]), ("c1", [])])
def test_bench_reference_arm_line(mesh, extra):
    """`bench.py --impl reference` end to end on small cases: one JSON line with the contract's keys,
    the reference kind, the rank count used and the same SAMPLING= as the GPU arm's timed runs."""
    import json
    import sys

    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--ref-mesh", mesh,
           "--ref-ranks", "2", "--steps", "2", "--warmup", "3"] + extra
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, start_new_session=True)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "RK-stage cell-updates/s" and line["value"] > 0
    assert line["steps"] == 2 and line["warmup"] == 3 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] == 2
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["ranks"] == 2 and line["config"]["sampling"] == 1_000_000_000
    assert line["config"]["cells"] == (8 ** 3 * 6 if mesh == "c3" else 64 * 32 * 2)
