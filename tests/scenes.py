"""Seeded scenes shared by the parity tests, and comparison helpers."""
from __future__ import annotations

import numpy as np

from aquarius_b200 import _abi


def ball_drop(size=(16, 16, 16), pool=0.2, center=(0.5, 0.65, 0.5), radius=0.15, dt=0.01, phase_ball=0, **kw):
    """The reference's ball-drop scene family: a pool filling y < pool plus a
    sphere, in the reference's normalised [0,1] coordinates."""
    vols = [dict(shape="box", min=(0, 0, 0), max=(1, pool, 1), phase=0),
            dict(shape="sphere", center=center, radius=radius, phase=phase_ball)]
    return _abi.make_config(size, vols, timestep=dt, **kw)


# name -> config; sizes the CPU oracle finishes in well under a second per step
SCENES = {
    "cfg1_16": lambda **kw: ball_drop((16, 16, 16), **kw),
    "cfg1_24": lambda **kw: ball_drop((24, 24, 24), **kw),
    "aniso": lambda **kw: ball_drop((20, 16, 24), pool=0.3, center=(0.4, 0.7, 0.55), radius=0.2, **kw),
    "cfg2_32": lambda **kw: ball_drop((32, 32, 32), pool=0.3, center=(0.5, 0.7, 0.5), radius=0.12, dt=0.005, **kw),
    "multi_16": lambda **kw: ball_drop((16, 16, 16), phase_ball=1, diffusion_coeff=0.01, **kw),
}


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    if den == 0:
        return float(num)
    return float(num / den)


def by_original(arr, sort_index):
    """Reorders a [k][N] (or [N]) sorted-particle array to pre-sort order."""
    arr = np.asarray(arr)
    out = np.empty_like(arr)
    out[..., sort_index] = arr
    return out
