"""Ink particles through the C ABI: the reference's switched-off ink path
(initInkRenderer, transferToInkParticles + moveInkParticles,
Fluid/Fluid_3D_FLIP.cu:600-725).

Seeding is host arithmetic over the replayed rand() sequence and must match
bit for bit; the advance is float G2P + RK3 and must match within relative
L2 1e-5 when both sides start from the same grids and ink (teacher forcing).
"""
import numpy as np
import pytest

import aquarius_b200 as aq
from golden_check import FLOAT_TOL, INK_SCENES, load_ink, replay_ink
from oracle_binding import Oracle, RefFluid, ref_available
from scenes import SCENES, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scene", ["cfg1_16", "aniso", "multi_16", "cfg1_24"])
def test_ink_seeding_matches_oracle(scene):
    cfg = SCENES[scene]()
    f, o = aq.Fluid(cfg), Oracle(cfg)
    assert f.ink_count == 0
    n = f.enable_ink()
    assert n == o.enable_ink() > 0
    assert f.enable_ink() == n  # seeded once
    a, b = f.get_ink(), o.get_ink()
    np.testing.assert_array_equal(a["position"], b["position"])
    assert not a["velocity"].any()


def test_ink_seeding_does_not_depend_on_steps_taken():
    """The ink continues the seeding's rand() sequence, which the steps never
    draw from: enabling it later seeds the same ink."""
    cfg = SCENES["cfg1_16"]()
    f = aq.Fluid(cfg)
    f.step(3)
    f.enable_ink()
    o = Oracle(cfg)
    o.enable_ink()
    np.testing.assert_array_equal(f.get_ink()["position"], o.get_ink()["position"])


def test_ink_calls_before_enable_fail():
    f = aq.Fluid(SCENES["cfg1_16"]())
    with pytest.raises(aq.AquariusError):
        f.ink_advance()
    with pytest.raises(aq.AquariusError):
        f.get_ink()


@pytest.mark.parametrize("scene,steps", [("cfg1_16", 6), ("aniso", 5), ("multi_16", 5), ("cfg1_24", 4)])
def test_ink_advance_teacher_forced(scene, steps):
    cfg = SCENES[scene]()
    o = Oracle(cfg)
    o.enable_ink()
    o.step(steps)  # the oracle's steps advance the ink too
    st = o.get_state()
    ink = o.get_ink()
    f = aq.Fluid(cfg)
    f.enable_ink()
    f.upload_state(st)
    f.set_ink(ink["position"], ink["velocity"])
    f.ink_advance()
    o.ink_advance()
    a, b = f.get_ink(), o.get_ink()
    assert np.abs(b["velocity"]).max() > 0
    for k in ("position", "velocity"):
        e = rel_l2(a[k], b[k])
        assert e <= FLOAT_TOL, (k, e)


@pytest.mark.parametrize("graph", [True, False])
def test_step_advances_ink_like_the_stages(graph):
    """A step with ink on (graph or eager) ends with the ink advance: equal,
    bit for bit, to the eight stages run one by one (the last one advances
    the ink)."""
    cfg = SCENES["cfg1_16"]()
    a, b = aq.Fluid(cfg), aq.Fluid(cfg)
    a.set_graph_mode(graph)
    for x in (a, b):
        x.enable_ink()
    a.step(3)
    for _ in range(3):
        for k in range(1, 9):
            b.run_stage(k)
    ia, ib = a.get_ink(), b.get_ink()
    for k in ("position", "velocity"):
        np.testing.assert_array_equal(ia[k], ib[k], err_msg=k)
    assert np.abs(ia["velocity"]).max() > 0


def test_step_with_ink_tracks_oracle():
    """One whole step from the same state and ink: the ink inherits the
    step's float differences, so the bound is the per-step one times ten."""
    cfg = SCENES["cfg1_16"]()
    o = Oracle(cfg)
    o.enable_ink()
    o.step(4)
    f = aq.Fluid(cfg)
    f.enable_ink()
    f.upload_state(o.get_state())
    ink = o.get_ink()
    f.set_ink(ink["position"], ink["velocity"])
    f.step(1)
    o.step(1)
    a, b = f.get_ink(), o.get_ink()
    for k in ("position", "velocity"):
        e = rel_l2(a[k], b[k])
        assert e <= 10 * FLOAT_TOL, (k, e)


def test_launch_count_includes_ink():
    cfg = SCENES["cfg1_16"]()
    f = aq.Fluid(cfg)
    f.step(1)
    before = f.launches_per_step()
    f.enable_ink()
    f.step(1)
    assert f.launches_per_step() == before + 1


@pytest.mark.parametrize("scene", INK_SCENES)
def test_library_ink_against_reference_fixtures(scene):
    data = load_ink()
    if data is None:
        pytest.skip("fixture missing")

    def set_grids(f, vel, nvel):
        f.upload_state({"velocity": vel, "new_velocity": nvel})

    res = replay_ink(data, scene, aq.Fluid, set_grids)
    assert res["count"][0] == res["count"][1]
    assert res["sample_equal"] and res["sha_match"]
    for s, ep, ev in res["steps"]:
        assert ep <= FLOAT_TOL and ev <= FLOAT_TOL, (s, ep, ev)


@pytest.mark.skipif(not ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("scene", ["cfg1_16", "multi_16"])
def test_ink_against_live_reference(scene):
    cfg = SCENES[scene]()
    r = RefFluid(cfg)
    n = r.enable_ink()
    f = aq.Fluid(cfg)
    assert f.enable_ink() == n
    np.testing.assert_array_equal(f.get_ink()["position"], r.get_ink()["position"])
    for _ in range(3):
        r.step(1)
        st = r.get_state(["velocity", "new_velocity"])
        ink = r.get_ink()
        f.upload_state(st)
        f.set_ink(ink["position"], ink["velocity"])
        f.ink_advance()
        r.ink_advance()
        a, b = f.get_ink(), r.get_ink()
        for k in ("position", "velocity"):
            e = rel_l2(a[k], b[k])
            assert e <= FLOAT_TOL, (k, e)
    r.close()
