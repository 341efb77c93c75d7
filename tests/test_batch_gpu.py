"""Scene batches on the GPU: every scene inside a batch must evolve bit for
bit as the same scene stepped alone (aq_fluid with the default Jacobi plan),
in fixed and residual solve modes, with scenes of uneven anisotropic sizes,
scenes whose residual solves stop at different sweep counts, and a scene
without fluid."""
import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi
from aquarius_b200.scenes import batch_configs

pytestmark = pytest.mark.gpu

FIELDS = ["position", "velocity_p", "velocity", "new_velocity", "pressure", "divergence", "particle_count_cell",
          "has_velocity", "density", "content", "cell_start", "cell_end", "particle_hash", "sort_index"]


def _mixed_configs(**solver):
    cs = batch_configs(5, seed=11, sizes=(12, 16, 20, 24), timestep=0.01, **solver)
    # a scene without fluid
    empty = _abi.make_config((16, 12, 8), [], **{k: getattr(cs[0], k) for k in (
        "timestep", "solve_mode", "pressure_init", "pressure_iterations", "rel_residual", "max_iterations",
        "check_interval")})
    return cs[:2] + [empty] + cs[2:]


def _assert_scene_equal(batch, s, alone):
    a = batch.download_scene(s, FIELDS)
    b = alone.download_state(FIELDS)
    for k in FIELDS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"scene {s} field {k}")
    assert a["physical_time"] == pytest.approx(b["physical_time"])


@pytest.mark.parametrize("solver", [
    dict(solve_mode=_abi.SOLVE_FIXED, pressure_init=_abi.PRESSURE_CARRY, pressure_iterations=37),
    dict(solve_mode=_abi.SOLVE_FIXED, pressure_init=_abi.PRESSURE_ZERO, pressure_iterations=40),
    dict(solve_mode=_abi.SOLVE_RESIDUAL, pressure_init=_abi.PRESSURE_ZERO, rel_residual=1e-3, max_iterations=400,
         check_interval=20),
    dict(solve_mode=_abi.SOLVE_RESIDUAL, pressure_init=_abi.PRESSURE_CARRY, rel_residual=1e-4, max_iterations=300,
         check_interval=10),
], ids=["fixed-carry-odd", "fixed-zero", "residual-zero", "residual-carry"])
def test_scene_in_batch_equals_scene_alone(solver):
    cfgs = _mixed_configs(**solver)
    steps = 4
    with aq.Batch(cfgs) as batch:
        assert batch.particle_counts[2] == 0
        for s, c in enumerate(cfgs):
            with aq.Fluid(c) as f:
                assert f.particleCount == batch.particle_counts[s]
                if s == 0:
                    _assert_scene_equal(batch, s, f)  # initial state
        batch.step(steps)
        batch.synchronize()
        iters = []
        for s, c in enumerate(cfgs):
            with aq.Fluid(c) as f:
                f.step(steps)
                f.synchronize()
                _assert_scene_equal(batch, s, f)
                sa, sb = batch.solve_stats(s), f.solve_stats()
                for k in ("iterations", "rel_residual", "b_norm", "fluid_cells", "converged", "blocks",
                          "total_sweeps", "total_blocks"):
                    assert sa[k] == sb[k], (s, k, sa[k], sb[k])
                iters.append(sa["iterations"])
        if solver["solve_mode"] == _abi.SOLVE_RESIDUAL:
            assert len(set(iters)) > 1  # scenes stopped at different sweep counts


def test_launch_shape_does_not_change_results():
    # sizes 12..160: one to five rows per warp, and two z blocks per row at 160
    cfgs = batch_configs(4, seed=3, sizes=(12, 20, 24), solve_mode=_abi.SOLVE_RESIDUAL, check_interval=20,
                         max_iterations=200, rel_residual=1e-3)
    cfgs.append(_abi.make_config((20, 12, 160), [dict(shape="box", min=(0, 0, 0), max=(1, 0.4, 1))],
                                 timestep=0.01, solve_mode=_abi.SOLVE_RESIDUAL, check_interval=20,
                                 max_iterations=200, rel_residual=1e-3, pressure_init=_abi.PRESSURE_ZERO))
    out = []
    for m, planes, pipe in ((1, 1, False), (64, 2, False), (3, 4, True), (64, 8, False), (64, 8, True)):
        with aq.Batch(cfgs) as b:
            b.set_grid_multiple(m)
            b.set_sweep_plan(planes, pipe)
            assert b.sweep_plan() == (planes, pipe)
            b.step(3)
            out.append([b.download_scene(s, ["position", "pressure"]) for s in range(len(cfgs))])
    for run in out[1:]:
        for a, b in zip(out[0], run):
            for k in ("position", "pressure"):
                np.testing.assert_array_equal(a[k], b[k])
    with aq.Fluid(cfgs[-1]) as f:
        f.step(3)
        np.testing.assert_array_equal(f.download_state(["pressure"])["pressure"], out[0][-1]["pressure"])


def test_batch_autotune_keeps_results():
    # zero-init pressure: the sweeps the tuner runs on the current systems do
    # not carry into the next step, so the tuned batch must stay bitwise equal
    cfgs = batch_configs(6, seed=9, sizes=(16, 24, 32), solve_mode=_abi.SOLVE_FIXED, pressure_iterations=30,
                         pressure_init=_abi.PRESSURE_ZERO)
    with aq.Batch(cfgs) as b, aq.Batch(cfgs) as ref:
        b.step(1)
        ref.step(1)
        r = b.autotune(20)
        assert r["x_planes"] in (1, 2, 4, 8) and r["sweep_us"] > 0
        assert b.sweep_plan() == (r["x_planes"], r["pipelined"])
        b.step(2)
        ref.step(2)
        for s in range(len(cfgs)):
            x, y = b.download_scene(s, ["position", "pressure"]), ref.download_scene(s, ["position", "pressure"])
            for k in ("position", "pressure"):
                np.testing.assert_array_equal(x[k], y[k])


def test_batch_launch_counts_and_benchmark():
    cfgs = batch_configs(6, seed=5, sizes=(16, 32), solve_mode=_abi.SOLVE_RESIDUAL, check_interval=20,
                         max_iterations=200)
    with aq.Batch(cfgs) as b:
        b.step(2)
        per_step, per_block = b.launch_counts()
        assert per_block == 20 + 3
        assert per_step == 6 + 5 + 4
        r = b.benchmark_pressure(40)
        assert r["ms"] > 0
        assert 0 < r["cells_per_sweep"] <= b.totals()["cells"]
