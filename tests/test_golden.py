"""CPU oracle against fixtures recorded from the reference's own kernels
(tests/golden/make_golden.py, run on a GPU with oracle/_ref built).

This pins the oracle: every stage of the first steps of three seeded scenes,
plus race-free settings of the reference's in-place kernels."""
import json

import numpy as np
import pytest

from golden_check import FLOAT_TOL, GOLDEN, INK_SCENES, judge, load, load_ink, replay, replay_ink, replay_special
from oracle_binding import Oracle

SCENES_STEPS = [("cfg1_16", 2), ("aniso", 1), ("multi_16", 1)]


def test_texture_probe_is_clamp():
    """The reference's tex3D with addressMode[1,2] left at the zero enum and
    unnormalised coordinates clamps on B200: Neumann walls on all faces."""
    p = json.loads((GOLDEN / "texture_probe.json").read_text())
    for k in ("x_low", "x_high", "y_low", "y_high", "z_low", "z_high"):
        assert p[k] == "clamp", (k, p[k])


@pytest.mark.parametrize("scene,steps", SCENES_STEPS)
def test_oracle_against_reference_fixtures(scene, steps):
    data = load(scene)
    if data is None:
        pytest.skip("fixture missing")
    directional = []
    res = replay(data, Oracle, steps, directional=directional)
    assert judge(res) == []
    # exactness where the reference does not race
    for (s, k, f, kind, v) in res:
        if kind == "int_mismatch" and not (k == 7 and f == "has_velocity"):
            assert v == 0, (s, k, f)
    assert all(v == 0 for v in directional)


def test_oracle_against_race_free_reference_settings():
    res = replay_special(Oracle)
    if res is None:
        pytest.skip("fixture missing")
    for name, f, kind, v, lim in res:
        assert v <= lim, (name, f, kind, v)


def test_fixture_seeding_is_bit_exact():
    """Particle seeding (glibc rand() jitter) reproduces the reference."""
    for scene, _ in SCENES_STEPS:
        data = load(scene)
        from golden_check import config_from_bytes
        o = Oracle(config_from_bytes(data["config"]))
        st = o.get_state(["position", "fractions", "sort_index", "cell_start", "cell_end", "content"])
        for k in st:
            if k != "physical_time":
                np.testing.assert_array_equal(st[k], data[f"init/{k}"], err_msg=f"{scene} {k}")


@pytest.mark.parametrize("scene", INK_SCENES)
def test_oracle_ink_against_reference_fixtures(scene):
    """Ink particles (the reference's switched-off initInkRenderer /
    transferToInkParticles / moveInkParticles): seeding bit-exact, each
    recorded advance within the float tolerance."""
    data = load_ink()
    if data is None:
        pytest.skip("fixture missing")

    def set_grids(o, vel, nvel):
        o.set_state({"velocity": vel, "new_velocity": nvel})

    res = replay_ink(data, scene, Oracle, set_grids)
    assert res["count"][0] == res["count"][1]
    assert res["sample_equal"] and res["sha_match"]
    assert len(res["steps"]) >= 2
    for s, ep, ev in res["steps"]:
        assert ep <= FLOAT_TOL and ev <= FLOAT_TOL, (s, ep, ev)
