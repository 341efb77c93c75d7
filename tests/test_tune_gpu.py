"""The Jacobi plan autotuner: picks a plan, keeps results unchanged (every
plan computes the same iterates), and round-trips its JSON cache."""
import json

import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi
from scenes import SCENES

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_plan_and_caches_it(tmp_path):
    cfg = SCENES["cfg2_32"](pressure_iterations=50)
    f = aq.Fluid(cfg)
    f.step(2)
    path = tmp_path / "tune.json"
    r = f.autotune(64, path)
    assert r["candidates"] >= 3 and not r["from_cache"]
    assert f.jacobi_plan() == r["plan"] and r["sweep_us"] > 0
    data = json.loads(path.read_text())
    assert len(data) == 1 and list(data.values())[0][:3] == list(r["plan"])
    g = aq.Fluid(cfg)
    g.step(1)
    r2 = g.autotune(64, path)
    assert r2["from_cache"] and r2["plan"] == r["plan"] and g.jacobi_plan() == r["plan"]


def test_tuned_plan_gives_identical_steps():
    cfg = SCENES["cfg2_32"](solve_mode=_abi.SOLVE_RESIDUAL, max_iterations=400, check_interval=40)
    a, b = aq.Fluid(cfg), aq.Fluid(cfg)
    a.step(2)
    b.step(2)
    b.autotune(64)
    sa = a.download_state(["pressure"])
    b.upload_state(sa)  # the tuner's trial sweeps advanced b's iterate
    a.step(2)
    b.step(2)
    x, y = a.download_state(), b.download_state()
    for k in x:
        if k != "physical_time":
            np.testing.assert_array_equal(x[k], y[k], err_msg=k)
