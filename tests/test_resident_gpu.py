"""The resident Jacobi plan (rows 4: the whole solve in one cooperative
launch, each CTA holding a tile and a K-cell halo in shared memory, halos
exchanged through L2 every K sweeps) against the one-sweep-per-launch plans
and the CPU oracle.  Temporal blocking with redundant halo work recomputes
exactly what K global sweeps compute, in the same order per cell, so the
iterates must be bit for bit those of the flat sweep (jacobiImpl,
Fluid/Fluid_3D_kernels.cu:460-505, race-free reading)."""
import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi
from oracle_binding import Oracle
from scenes import SCENES, ball_drop, rel_l2

pytestmark = pytest.mark.gpu

RESIDENT = [(4, 4, s) for s in range(6)]


def _system(cfg, steps=3):
    o = Oracle(cfg)
    o.step(steps)
    for k in range(1, 5):
        o.stage(k)
    st = o.get_state()
    return o, st


def _solve(cfg, st, plan):
    with aq.Fluid(cfg) as f:
        if plan is not None:
            f.set_jacobi_plan(*plan)
        f.upload_state(st)
        f.run_stage(_abi.STAGE_PRESSURE)
        return f.download_state(["pressure"])["pressure"], f.solve_stats()


def test_division_by_six_matches_ieee_on_every_float():
    import ctypes as ct
    lib = aq.load_library()
    bad = ct.c_uint64(123)
    assert lib.aq_selfcheck_division(0, ct.byref(bad)) == 0
    assert bad.value == 0


@pytest.mark.parametrize("sweeps", [1, 3, 4, 61, 100])
def test_resident_fixed_equals_flat(sweeps):
    cfg = SCENES["cfg2_32"](pressure_init=_abi.PRESSURE_ZERO, pressure_iterations=sweeps)
    o, st = _system(cfg)
    p0, s0 = _solve(cfg, st, (1, 0, 1))
    for plan in RESIDENT:
        p, s = _solve(cfg, st, plan)
        np.testing.assert_array_equal(p, p0, err_msg=str(plan))
        assert s["iterations"] == sweeps
        assert s["rel_residual"] == pytest.approx(s0["rel_residual"], rel=1e-9), plan
    o.stage(_abi.STAGE_PRESSURE)
    assert rel_l2(p0, o.get_state(["pressure"])["pressure"]) <= 1e-5
    o.close()


def test_resident_residual_mode_equals_list_plan():
    cfg = SCENES["cfg2_32"](pressure_init=_abi.PRESSURE_ZERO, solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=1e-4,
                            max_iterations=800, check_interval=40)
    o, st = _system(cfg)
    p0, s0 = _solve(cfg, st, (1, 3, 1))
    for plan in RESIDENT:
        p, s = _solve(cfg, st, plan)
        assert s["iterations"] == s0["iterations"], plan
        np.testing.assert_array_equal(p, p0, err_msg=str(plan))
        assert s["rel_residual"] == pytest.approx(s0["rel_residual"], rel=1e-9), plan
    o.stage(_abi.STAGE_PRESSURE)
    assert s0["iterations"] == o.solve_stats()["iterations"]
    o.close()


@pytest.mark.parametrize("size,plan0", [((52, 50, 52), (2, 16, 16)), ((30, 28, 36), (1, 0, 1)),
                                        ((20, 16, 24), (1, 0, 1))])
def test_resident_on_ragged_grids(size, plan0):
    """Tiles that overhang the grid on every axis, carried pressure."""
    cfg = ball_drop(size, pool=0.3, center=(0.45, 0.7, 0.55), radius=0.2, pressure_iterations=57)
    o, st = _system(cfg, steps=4)
    p0, _ = _solve(cfg, st, plan0)
    for plan in [(4, 4, 0), (4, 4, 2), (4, 4, 4), (4, 4, 5)]:
        p, _ = _solve(cfg, st, plan)
        np.testing.assert_array_equal(p, p0, err_msg=str(plan))
    o.stage(_abi.STAGE_PRESSURE)
    assert rel_l2(p0, o.get_state(["pressure"])["pressure"]) <= 1e-5
    o.close()


def test_resident_walks_tiles_when_they_outnumber_the_ctas():
    """128^3 pool in 8x16x16 tiles: ~380 active tiles for at most one CTA
    per SM, so each CTA reloads several tiles per block from L2."""
    cfg = SCENES["cfg2_32"](pressure_init=_abi.PRESSURE_ZERO, pressure_iterations=23)
    cfg.size_x = cfg.size_y = cfg.size_z = 128
    with aq.Fluid(cfg) as f:
        f.step(1)
        f.synchronize()
        st = f.download_state()
    p0, _ = _solve(cfg, st, (1, 3, 1))
    for plan in [(4, 4, 4), (4, 4, 3)]:
        p, _ = _solve(cfg, st, plan)
        np.testing.assert_array_equal(p, p0, err_msg=str(plan))


def test_resident_whole_steps_in_graph_match_list_plan():
    cfg = SCENES["cfg2_32"](pressure_init=_abi.PRESSURE_CARRY, solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=1e-4,
                            max_iterations=400, check_interval=20)
    out = {}
    for plan in [(1, 3, 1), (4, 4, 0), (4, 4, 2)]:
        with aq.Fluid(cfg) as f:
            f.set_jacobi_plan(*plan)
            f.step(5)
            f.synchronize()
            out[plan] = f.download_state(["pressure", "position", "new_velocity"])
    for plan in out:
        for k in out[plan]:
            if k != "physical_time":
                np.testing.assert_array_equal(out[plan][k], out[(1, 3, 1)][k], err_msg=f"{plan} {k}")


def test_resident_learned_start_matches_list_plan():
    net = aq.UNet(0, seed=7)
    cfg = SCENES["cfg2_32"](pressure_init=_abi.PRESSURE_LEARNED, solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=1e-4,
                            max_iterations=400, check_interval=40)
    out = {}
    for plan in [(1, 3, 1), (4, 4, 0)]:
        with aq.Fluid(cfg) as f:
            f.set_warm_start(net)
            f.set_jacobi_plan(*plan)
            f.step(3)
            f.synchronize()
            out[plan] = (f.download_state(["pressure"])["pressure"], f.solve_stats())
    (pa, sa), (pb, sb) = out[(1, 3, 1)], out[(4, 4, 0)]
    np.testing.assert_array_equal(pb, pa)
    assert sb["iterations"] == sa["iterations"] and sb["warm_start"] == sa["warm_start"]
    net.close()
