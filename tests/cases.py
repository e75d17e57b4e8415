"""Test cases shared by the CPU and GPU suites: small seeded meshes of the three benchmark
families, flow settings, and consistent perturbed flow states."""
from __future__ import annotations

import dataclasses
from typing import Dict

import numpy as np

from euler3d_b200 import meshgen as mg
from euler3d_b200.solver import FlowConfig, Mesh

STATE_KEYS = ("rho", "u", "v", "w", "p", "E", "H", "M")


@dataclasses.dataclass
class Case:
    name: str
    make: object          # () -> RawMesh
    mach: float
    aoa: float
    cfl: float

    def raw(self) -> mg.RawMesh:
        return self.make()

    def flow(self, **kw) -> FlowConfig:
        return FlowConfig(mach=self.mach, aoa=self.aoa, cfl=self.cfl, **kw)


CASES = {
    "channel": Case("channel", lambda: mg.bump_channel(16, 8, 2), 0.5, 0.0, 1.5),
    "channel_supersonic": Case("channel_supersonic", lambda: mg.bump_channel(16, 8, 2, seed=5), 1.5, 2.0, 0.8),
    "ogrid": Case("ogrid", lambda: mg.biconvex_ogrid(24, 12, 2), 0.8, 1.25, 1.2),
    "tets": Case("tets", lambda: mg.bump_box_tets(5), 0.6, 0.0, 1.0),
    "pyramids": Case("pyramids", lambda: mg.bump_box_pyramids(4), 0.6, 2.0, 1.0),
    "c1": Case("c1", lambda: mg.bump_channel(), 0.5, 0.0, 1.5),
}

_prepared: Dict[str, dict] = {}


def prepared(name: str) -> dict:
    """Prepared mesh arrays (product preprocessing, reference numbering), cached per session."""
    if name not in _prepared:
        _prepared[name] = Mesh.from_raw(CASES[name].raw()).arrays()
    return _prepared[name]


def perturbed_state(arrays: dict, flow: FlowConfig, seed: int, amp: float = 0.05,
                    ghost_mach_range=(0.3, 1.7)) -> Dict[str, np.ndarray]:
    """A consistent flow state (E, H from rho, u, p) a few percent off the freestream; ghost Mach
    numbers span sub- and supersonic values so every farfield branch is taken."""
    n = int(arrays["n_cells"])
    t = n + int(arrays["n_faces"]) - int(arrays["n_faces_int"])
    rng = np.random.default_rng(seed)
    g = flow.gamma
    a = np.deg2rad(flow.aoa)
    uinf = flow.mach * np.sqrt(g)
    rho = 1.0 + amp * rng.uniform(-1, 1, t)
    p = 1.0 + amp * rng.uniform(-1, 1, t)
    u = uinf * np.cos(a) + amp * uinf * rng.uniform(-1, 1, t) + 0.05 * rng.uniform(-1, 1, t)
    v = uinf * np.sin(a) + amp * rng.uniform(-1, 1, t)
    w = amp * rng.uniform(-1, 1, t)
    q2 = u * u + v * v + w * w
    E = p / ((g - 1) * rho) + q2 / 2.0
    H = E + p / rho
    M = np.sqrt(g * (p / rho)) / np.sqrt(q2)
    M[n:] = rng.uniform(*ghost_mach_range, t - n)
    return {"rho": rho, "u": u, "v": v, "w": w, "p": p, "E": E, "H": H, "M": M}
