"""Parity of the CUDA library against the CPU oracle, through the C ABI.

Teacher forcing: every stage starts both implementations from the same
state (the oracle's), so differences do not compound.  Integer/index outputs
(hashes, permutation, cell tables, counts, cell types, has-velocity bits)
must match bit for bit; float fields within relative L2 1e-5.
"""
import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi
from oracle_binding import Oracle
from scenes import SCENES, ball_drop, by_original, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative L2 per step (float fields)
INT_FIELDS = ["content", "particle_count_cell", "cell_start", "cell_end", "particle_hash", "sort_index"]


def make_pair(cfg):
    o = Oracle(cfg)
    f = aq.Fluid(cfg)
    assert f.particleCount == o.n
    return f, o


def warm(o, steps):
    for _ in range(steps):
        o.step(1)


@pytest.mark.parametrize("scene", ["cfg1_16", "cfg1_24", "aniso", "multi_16"])
def test_init_matches_oracle(scene):
    cfg = SCENES[scene]()
    f, o = make_pair(cfg)
    a, b = f.download_state(), o.get_state()
    # host seeding reproduces the glibc rand() sequence: positions bit-exact
    np.testing.assert_array_equal(a["position"], b["position"])
    np.testing.assert_array_equal(a["fractions"], b["fractions"])
    for k in ["content", "cell_start", "cell_end", "sort_index", "particle_hash"]:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in ["velocity", "new_velocity", "density"]:
        assert rel_l2(a[k], b[k]) <= TOL, k


def _stage_inputs(scene, steps, upto):
    """Oracle state after `steps` full steps and stages 1..upto-1 of the next."""
    cfg = SCENES[scene]()
    o = Oracle(cfg)
    warm(o, steps)
    for k in range(1, upto):
        o.stage(k)
    return cfg, o


def _inject(cfg, state):
    f = aq.Fluid(cfg)
    f.upload_state(state)
    return f


@pytest.mark.parametrize("scene,steps", [("cfg1_16", 6), ("cfg1_24", 4), ("aniso", 5), ("multi_16", 5)])
def test_sort_is_bit_exact(scene, steps):
    cfg, o = _stage_inputs(scene, steps, 2)  # after G2P+advect: positions not yet sorted
    st = o.get_state()
    f = _inject(cfg, st)
    f.run_stage("sort")
    o.stage(_abi.STAGE_SORT)
    a, b = f.download_state(), o.get_state()
    for k in ["sort_index", "cell_start", "cell_end", "particle_hash", "position", "velocity_p"]:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    # the permutation is the stable sort of the cell keys
    keys = b["particle_hash"][np.argsort(b["sort_index"])]
    np.testing.assert_array_equal(np.argsort(keys, kind="stable"), b["sort_index"])


@pytest.mark.parametrize("scene,steps", [("cfg1_16", 6), ("cfg1_24", 4), ("aniso", 5), ("multi_16", 5)])
def test_g2p_advect(scene, steps):
    cfg, o = _stage_inputs(scene, steps, 1)
    f = _inject(cfg, o.get_state())
    f.run_stage("g2p_advect")  # fused with the sort
    o.stage(_abi.STAGE_G2P_ADVECT)
    o.stage(_abi.STAGE_SORT)
    a, b = f.download_state(), o.get_state()
    for k in ["position", "velocity_p", "fractions"]:
        pa = by_original(a[k], a["sort_index"])
        pb = by_original(b[k], b["sort_index"])
        assert rel_l2(pa, pb) <= TOL, (k, rel_l2(pa, pb))
    # the sort of the library's own positions is exact
    keys = a["particle_hash"][np.argsort(a["sort_index"])]
    np.testing.assert_array_equal(np.argsort(keys, kind="stable"), a["sort_index"])


STAGE_OUT = {
    _abi.STAGE_P2G: ["velocity", "new_velocity", "density", "volume_fractions", "new_volume_fractions"],
    _abi.STAGE_DIVERGENCE: ["divergence"],
    _abi.STAGE_PRESSURE: ["pressure"],
    _abi.STAGE_PROJECT: ["new_velocity"],
    _abi.STAGE_EXTRAPOLATE: ["new_velocity"],
    _abi.STAGE_DIFFUSE: ["new_volume_fractions"],
}
STAGE_INT = {
    _abi.STAGE_P2G: ["content"],
    _abi.STAGE_DIVERGENCE: ["particle_count_cell"],
    _abi.STAGE_PROJECT: ["has_velocity"],
    _abi.STAGE_EXTRAPOLATE: ["has_velocity"],
}


@pytest.mark.parametrize("scene,steps", [("cfg1_16", 6), ("cfg1_24", 4), ("aniso", 5), ("multi_16", 5),
                                         ("cfg2_32", 3)])
@pytest.mark.parametrize("stage", [_abi.STAGE_P2G, _abi.STAGE_DIVERGENCE, _abi.STAGE_PRESSURE,
                                   _abi.STAGE_PROJECT, _abi.STAGE_EXTRAPOLATE, _abi.STAGE_DIFFUSE])
def test_grid_stage(scene, steps, stage):
    cfg, o = _stage_inputs(scene, steps, stage)
    f = _inject(cfg, o.get_state())
    f.run_stage(stage)
    o.stage(stage)
    a, b = f.download_state(), o.get_state()
    for k in STAGE_INT.get(stage, []):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in STAGE_OUT[stage]:
        if np.linalg.norm(b[k]) == 0 and np.linalg.norm(a[k]) == 0:
            continue
        e = rel_l2(a[k], b[k])
        assert e <= TOL, (k, e)


@pytest.mark.parametrize("scene", ["cfg1_16", "cfg1_24", "multi_16"])
def test_full_steps_teacher_forced(scene):
    """Each step starts both from the oracle's state; compare after the step."""
    cfg = SCENES[scene]()
    o = Oracle(cfg)
    f = aq.Fluid(cfg)
    for step in range(8):
        f.upload_state(o.get_state())
        f.step(1)
        o.step(1)
        a, b = f.download_state(), o.get_state()
        for k in ["pressure", "new_velocity", "velocity", "divergence", "density"]:
            e = rel_l2(a[k], b[k])
            assert e <= TOL, (step, k, e)
        for k in ["position", "velocity_p"]:
            e = rel_l2(by_original(a[k], a["sort_index"]), by_original(b[k], b["sort_index"]))
            assert e <= TOL, (step, k, e)
        assert abs(a["physical_time"] - b["physical_time"]) < 1e-9


def test_graph_equals_eager_stages():
    """The captured step graph and the eager stage sequence are bitwise equal."""
    cfg = SCENES["cfg1_24"]()
    f1, f2 = aq.Fluid(cfg), aq.Fluid(cfg)
    for _ in range(3):
        f1.step(1)
        for k in range(1, 9):
            f2.run_stage(k)
    a, b = f1.download_state(), f2.download_state()
    for k in a:
        if k == "physical_time":
            continue
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_deterministic_runs():
    cfg = SCENES["cfg2_32"]()
    states = []
    for _ in range(2):
        f = aq.Fluid(cfg)
        f.step(5)
        states.append(f.download_state())
    for k in states[0]:
        if k != "physical_time":
            np.testing.assert_array_equal(states[0][k], states[1][k], err_msg=k)


def test_free_running_plausibility():
    """Free-running (no teacher forcing): chaotic divergence is allowed, but
    global quantities must track the oracle."""
    cfg = SCENES["cfg1_24"]()
    f, o = make_pair(cfg)
    f.step(20)
    o.step(20)
    a, b = f.download_state(), o.get_state()
    fa, fb = (a["content"] == 1).sum(), (b["content"] == 1).sum()
    assert abs(int(fa) - int(fb)) <= 0.02 * fb
    ke_a = float((a["velocity_p"].astype(np.float64) ** 2).sum())
    ke_b = float((b["velocity_p"].astype(np.float64) ** 2).sum())
    assert abs(ke_a - ke_b) <= 0.05 * ke_b
    com_a, com_b = a["position"].mean(axis=1), b["position"].mean(axis=1)
    assert np.abs(com_a - com_b).max() < 0.02 * cfg.domain_size


def test_residual_mode_graph_matches_eager_and_oracle():
    cfg = SCENES["cfg2_32"](solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=1e-4, max_iterations=2000,
                            check_interval=40, pressure_init=_abi.PRESSURE_ZERO)
    o = Oracle(cfg)
    warm(o, 3)
    st = o.get_state()
    f1, f2 = aq.Fluid(cfg), aq.Fluid(cfg)
    f1.upload_state(st)
    f2.upload_state(st)
    f1.step(1)                     # graph with a conditional while node
    for k in range(1, 9):          # eager: host reads the residual per block
        f2.run_stage(k)
    o.step(1)
    s1, s2, so = f1.solve_stats(), f2.solve_stats(), o.solve_stats()
    assert s1["iterations"] == s2["iterations"] == so["iterations"]
    assert s1["iterations"] % 40 == 0
    assert s1["converged"] or s1["iterations"] >= 2000
    if s1["converged"]:
        assert s1["rel_residual"] <= 1e-4
    assert abs(s1["rel_residual"] - so["rel_residual"]) <= 1e-6 + 1e-3 * so["rel_residual"]
    a, b = f1.download_state(["pressure"]), f2.download_state(["pressure"])
    np.testing.assert_array_equal(a["pressure"], b["pressure"])
    assert rel_l2(a["pressure"], o.get_state(["pressure"])["pressure"]) <= TOL


def test_fixed_mode_reports_residual():
    cfg = SCENES["cfg1_16"]()
    f, o = make_pair(cfg)
    f.step(2)
    o.step(2)
    s, so = f.solve_stats(), o.solve_stats()
    assert s["iterations"] == 100 == so["iterations"]
    assert s["rel_residual"] == pytest.approx(so["rel_residual"], rel=1e-3)
    assert s["fluid_cells"] == so["fluid_cells"]


def test_pcg_reference_solves_the_system():
    cfg = SCENES["cfg2_32"]()
    o = Oracle(cfg)
    warm(o, 3)
    for k in range(1, 5):
        o.stage(k)
    f = _inject(cfg, o.get_state())
    r = f.pcg_reference(rel_tol=1e-12, want_pressure=True)
    assert r["residual"] <= 1e-12
    # check A x = b independently in numpy (FP64)
    st = o.get_state()
    sx, sy, sz = cfg.size_x, cfg.size_y, cfg.size_z
    fluid = (st["content"].reshape(sx + 1, sy + 1, sz + 1)[:sx, :sy, :sz] == 1)
    p = np.where(fluid, r["pressure"].reshape(sx, sy, sz).astype(np.float64), 0.0)
    b = np.where(fluid, -(st["divergence"] * st["density"]).reshape(sx, sy, sz).astype(np.float64), 0.0)
    Ap = np.zeros_like(p)
    nin = np.zeros_like(p)
    for ax in range(3):
        for sh in (1, -1):
            q = np.roll(p, sh, axis=ax)
            valid = np.ones_like(p, dtype=bool)
            idx = [slice(None)] * 3
            idx[ax] = 0 if sh == 1 else -1
            valid[tuple(idx)] = False
            Ap -= np.where(valid, q, 0.0)
            nin += valid
    Ap += nin * p
    res = np.linalg.norm(np.where(fluid, b - Ap, 0.0)) / np.linalg.norm(b)
    assert res < 1e-5  # float32 rounding of the returned solution


def test_host_buffer_step_matches_device_step():
    cfg = SCENES["cfg1_16"]()
    f1, f2 = aq.Fluid(cfg), aq.Fluid(cfg)
    n = f1.particleCount
    pos = np.zeros((3, n), np.float32)
    vel = np.zeros((3, n), np.float32)
    f1.step(3)
    f2.step_host(3, None, None, pos, vel)
    a = f1.download_state(["position", "velocity_p"])
    np.testing.assert_array_equal(a["position"], pos)
    np.testing.assert_array_equal(a["velocity_p"], vel)
    # round trip of host buffers is the identity on the state
    f2.step_host(0, pos, vel, pos, vel)
    np.testing.assert_array_equal(a["position"], pos)


def test_empty_scene_steps():
    cfg = _abi.make_config((16, 16, 16), [])
    f = aq.Fluid(cfg)
    assert f.particleCount == 0
    f.step(3)
    s = f.download_state(["pressure", "content"])
    assert not s["pressure"].any()
    assert f.physicalTime == pytest.approx(3 * cfg.timestep)


def test_upload_rejects_positions_outside_domain():
    cfg = SCENES["cfg1_16"]()
    f = aq.Fluid(cfg)
    st = f.download_state(["position"])
    st["position"][0, 0] = -1.0
    with pytest.raises(aq.AquariusError):
        f.upload_state(st)


def test_reference_api_surface():
    fc = aq.FluidConfig()
    fc.FLIP.sizeX = fc.FLIP.sizeY = fc.FLIP.sizeZ = 24
    fl = aq.Fluid()
    fl.init(fc)
    assert fl.getCenter() == (5.0, 5.0, 5.0)
    assert fl.getContainerSize() == 10.0
    fl.simulationStep()
    fl.draw(None)
    assert fl.physicalTime == pytest.approx(0.033)


def test_full_size_invariants():
    """BASELINE config-2 size (128^3, 5.2M particles): size-independent checks
    after a few steps — sortedness, cell tables, permutation, bounds."""
    cfg = ball_drop((128, 128, 128), pool=0.3, center=(0.5, 0.7, 0.5), radius=0.12, dt=0.005,
                    solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=1e-4, max_iterations=2000, check_interval=40)
    f = aq.Fluid(cfg)
    assert 5_200_000 < f.particleCount < 5_300_000
    f.step(3)
    s = f.download_state(["position", "particle_hash", "cell_start", "cell_end", "sort_index", "content",
                          "particle_count_cell"])
    n = f.particleCount
    h = s["particle_hash"]
    assert (np.diff(h) >= 0).all()
    assert np.array_equal(np.sort(s["sort_index"]), np.arange(n))
    occ = s["cell_start"] >= 0
    counts = np.where(occ, s["cell_end"] - s["cell_start"] + 1, 0)
    assert counts.sum() == n
    np.testing.assert_array_equal(np.bincount(h, minlength=counts.size), counts)
    np.testing.assert_array_equal(s["particle_count_cell"], np.where(occ, counts - 1, 0))
    L = cfg.domain_size
    hh = L / 128
    assert s["position"].min() >= hh / 4 - 1e-6 and s["position"].max() <= L - hh / 4 + 1e-5
    # positions -> cells with IEEE division match the hashes
    q = (s["position"] / np.float32(hh)).astype(np.int32)
    np.testing.assert_array_equal((q[0] * 128 + q[1]) * 128 + q[2], h)
    st = f.solve_stats()
    assert st["iterations"] > 0 and (st["converged"] or st["iterations"] >= 2000)


@pytest.mark.parametrize("mode", ["fixed", "residual"])
def test_jacobi_plans_agree(mode):
    """Every Jacobi plan (flat, persistent cooperative, temporally blocked)
    computes the same iterates: same arithmetic per cell, same order."""
    kw = dict(pressure_init=_abi.PRESSURE_ZERO)
    if mode == "residual":
        kw.update(solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=1e-4, max_iterations=800, check_interval=40)
    else:
        kw.update(pressure_iterations=61)
    cfg = SCENES["cfg2_32"](**kw)
    o = Oracle(cfg)
    warm(o, 3)
    for k in range(1, 5):
        o.stage(k)
    st = o.get_state()
    results = {}
    for plan in [(1, 0, 1), (1, 1, 1), (1, 0, 2), (2, 16, 16), (4, 32, 16), (1, 2, 8), (2, 2, 8), (3, 2, 8),
                 (4, 2, 8), (2, 2, 16), (4, 2, 16), (1, 3, 1)]:
        f = aq.Fluid(cfg)
        f.set_jacobi_plan(*plan)
        f.upload_state(st)
        f.run_stage(_abi.STAGE_PRESSURE)
        results[plan] = (f.download_state(["pressure"])["pressure"], f.solve_stats())
        f.close()
    p0, s0 = results[(1, 0, 1)]
    for plan, (p, s) in results.items():
        np.testing.assert_array_equal(p, p0, err_msg=str(plan))
        assert s["iterations"] == s0["iterations"], plan
        assert s["rel_residual"] == pytest.approx(s0["rel_residual"], rel=1e-9), plan
    o.stage(_abi.STAGE_PRESSURE)
    assert rel_l2(p0, o.get_state(["pressure"])["pressure"]) <= TOL
    assert s0["iterations"] == o.solve_stats()["iterations"]


@pytest.mark.parametrize("shape", [(40, 36, 52), (24, 20, 28)])
def test_cube_and_list_plans_match_flat_on_ragged_grids(shape):
    # tiles that overhang the grid on every axis, full steps in a graph
    vols = [dict(shape="box", min=(0, 0, 0), max=(1, 0.35, 1)),
            dict(shape="sphere", center=(0.45, 0.7, 0.55), radius=0.2)]
    cfg = _abi.make_config(shape, vols, timestep=0.01, pressure_init=_abi.PRESSURE_CARRY, pressure_iterations=57)
    ref = aq.Fluid(cfg)
    ref.step(3)
    a = ref.download_state(["pressure", "position", "new_velocity"])
    ref.close()
    for plan in [(2, 2, 8), (3, 2, 8), (4, 2, 8), (2, 2, 16), (4, 2, 16), (1, 3, 1)]:
        with aq.Fluid(cfg) as f:
            f.set_jacobi_plan(*plan)
            f.step(3)
            b = f.download_state(["pressure", "position", "new_velocity"])
        for k in ("pressure", "position", "new_velocity"):
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"{plan} {k}")


def test_persistent_step_graph_matches_flat():
    cfg = SCENES["cfg2_32"](solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=1e-4, max_iterations=400, check_interval=40)
    f1, f2 = aq.Fluid(cfg), aq.Fluid(cfg)
    f2.set_jacobi_plan(1, 1, 1)
    f1.step(4)
    f2.step(4)
    a, b = f1.download_state(), f2.download_state()
    for k in a:
        if k != "physical_time":
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
