"""Seeded scene sets for batches of independent ball-drop scenes.

The batch workload: n scenes whose grid sizes are drawn per axis from
{24, 32, 48, 64}, each a pool of random depth 0.1-0.4 plus 1-2 spheres of
radius 0.08-0.2 (fractions of the domain height, as the reference's
ballRadius) at random positions above the pool, 8 particles per fluid cell
from the reference seeding, one phase.  Everything else follows the
reference's FluidConfig defaults (Fluid/FluidConfig.cuh) except the solver
settings passed in.
"""
from __future__ import annotations

import numpy as np

from . import _abi

BATCH_SIZES = (24, 32, 48, 64)


def batch_configs(n_scenes: int = 256, seed: int = 2024, sizes=BATCH_SIZES, timestep: float = 0.01,
                  solve_mode: int = _abi.SOLVE_RESIDUAL, pressure_init: int = _abi.PRESSURE_ZERO,
                  pressure_iterations: int = 100, rel_residual: float = 1e-4, max_iterations: int = 2000,
                  check_interval: int = 40, device: int = 0) -> list:
    """Configs of a seeded scene set (see the module docstring)."""
    rng = np.random.RandomState(seed)
    out = []
    for i in range(n_scenes):
        sx, sy, sz = (int(rng.choice(sizes)) for _ in range(3))
        depth = float(rng.uniform(0.1, 0.4))
        vols = [dict(shape="box", min=(0.0, 0.0, 0.0), max=(1.0, depth, 1.0), phase=0)]
        for _ in range(int(rng.randint(1, 3))):
            r = float(rng.uniform(0.08, 0.2))
            # centre above the pool, inside the unit cube of relative coordinates
            cy = float(rng.uniform(min(depth + r, 0.95), 0.95))
            cx, cz = (float(rng.uniform(0.2, 0.8)) for _ in range(2))
            vols.append(dict(shape="sphere", center=(cx, cy, cz), radius=r, phase=0))
        out.append(_abi.make_config(
            (sx, sy, sz), vols, timestep=timestep, flip_coeff=0.95, particle_jitter=0.05, seed=1 + i,
            pressure_init=pressure_init, solve_mode=solve_mode, pressure_iterations=pressure_iterations,
            rel_residual=rel_residual, max_iterations=max_iterations, check_interval=check_interval,
            device=device))
    return out


def batch_desc(n_scenes: int, seed: int, sizes=BATCH_SIZES) -> str:
    return (f"{n_scenes} ball-drop scenes, sizes per axis from {list(sizes)} (seed {seed}), pool depth 0.1-0.4 "
            f"+ 1-2 spheres r 0.08-0.2, 8ppc, dt=0.01")
