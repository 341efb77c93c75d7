"""CPU oracle against fixtures recorded from the reference's own kernels
(tests/golden/make_golden.py, run on a GPU with oracle/_ref built).

This pins the oracle: every stage of the first steps of three seeded scenes,
plus race-free settings of the reference's in-place kernels."""
import json

import numpy as np
import pytest

from golden_check import (FLOAT_TOL, GOLDEN, INK_SCENES, judge, load, load_ink, replay, replay_ink, replay_special,
                          spreads)
from oracle_binding import Oracle, oracle_tex_linear

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
    assert judge(res, spreads().get(scene, {})) == []
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


def test_texture_filter_model_against_reference_probe():
    """The mesher samples its SDF through the texture unit (linear filter,
    x border).  Along one axis the weight is the fraction rounded half up to
    1/256, exactly; in 3D the oracle's model of the per-texel weight rounding
    reproduces the probe for most samples."""
    p = np.load(GOLDEN / "texture_linear_probe.npz")
    vals, coords, out = p["values"], p["coords"].astype(np.float64), p["out"]
    sweep = coords[:, 1] == 2.5
    sweep &= coords[:, 2] == 2.5
    x = coords[sweep, 0] - 0.5
    i = np.floor(x).astype(int)
    a = np.floor((x - i) * 256 + 0.5) / 256
    row = vals[2, 2].astype(np.float64)
    pred = (1 - a) * row[i] + a * row[np.minimum(i + 1, row.size - 1)]
    assert np.abs(pred - out[sweep]).max() < 1e-6
    got = oracle_tex_linear(vals, coords)
    err = np.abs(got - out)
    assert (err <= 1e-6).mean() >= 0.9
    assert err.max() <= 0.02


MESH_SCENES = [("cfg1_16", "ref_cfg1_16"), ("aniso", "ref_aniso")]


@pytest.mark.parametrize("scene,fixture", MESH_SCENES)
def test_oracle_mesh_against_reference_fixtures(scene, fixture):
    """Surface mesher (the reference's Mesher run on the recorded particles):
    the SDF within float rounding, the same occupied cubes, and the sampled
    records matched vertex by vertex (the texture unit's weights are only
    modelled, so a few vertices move by up to a tenth of a mesh cell)."""
    from mesh_check import match_records, record_aggregates, used_slots
    from scenes import SCENES, rel_l2

    mz = np.load(GOLDEN / "ref_mesh.npz")
    pos = np.load(GOLDEN / f"{fixture}.npz")[str(mz[f"{scene}/input"])]
    o = Oracle(SCENES[scene]())
    o.set_state({"position": pos})
    r = o.mesh()
    d = r["dims"]
    assert tuple(mz[f"{scene}/sdf_size"]) == d["sdf"] and tuple(mz[f"{scene}/mesh_size"]) == d["mesh"]
    assert np.allclose(mz[f"{scene}/cell"], [d["h_sdf"], d["h_mesh"]], rtol=0, atol=0)
    ref_sdf = mz[f"{scene}/sdf"].transpose(2, 1, 0)
    assert rel_l2(r["sdf"], ref_sdf) <= 1e-5
    assert np.abs(r["sdf"] - ref_sdf).max() <= 1e-4 * d["h_sdf"]
    cubes = int(mz[f"{scene}/cubes"])
    assert abs(r["cubes"] - cubes) <= 5e-4 * cubes
    agg = record_aggregates(r["records"])
    assert abs(agg["vertices"] - int(mz[f"{scene}/agg/vertices"])) <= 5e-4 * agg["vertices"]
    sample = mz[f"{scene}/sample"]
    pairs, un_a, _ = match_records(sample, r["records"], 0.25 * d["h_mesh"])
    assert len(pairs) >= 0.99 * len(sample)
    ra, rb = sample[pairs[:, 0]], r["records"][pairs[:, 1]]
    u = used_slots(ra)
    dp = np.abs(ra[..., :3] - rb[..., :3]).max(-1)[u] / d["h_mesh"]
    assert np.percentile(dp, 50) <= 1e-4 and np.percentile(dp, 99) <= 0.02 and dp.max() <= 0.1
    # Normals are central differences of the filtered SDF half a mesh cell
    # apart; where the SDF is flat (inside the fluid, on the mesh grid's
    # clipping faces) they follow the filter's rounding and may point anywhere.
    dn = np.abs(ra[..., 3:] - rb[..., 3:]).max(-1)[u]
    assert (dn <= 0.05).mean() >= 0.95


@pytest.mark.parametrize("method", ["pbf", "pcisph"])
def test_sph_oracle_against_reference_fixtures(method):
    """Particle-only solvers: seeding and the init's stable sort bit for bit,
    rest densities to float rounding, and every recorded step teacher-forced
    from the reference's own state (judge_sph_step's bounds)."""
    from golden_check import judge_sph_step, load_sph, sph_config_from_bytes, sph_fixture_state
    from oracle_binding import SphOracle
    from scenes import rel_l2

    data = load_sph()
    if data is None:
        pytest.skip("fixture missing")
    o = SphOracle(sph_config_from_bytes(data[f"{method}/config"]))
    assert (o.spacing, o.kernel_radius) == tuple(float(v) for v in data[f"{method}/info"])
    assert o.grid == tuple(int(v) for v in data[f"{method}/grid"])
    st = o.get_state()
    s0 = sph_fixture_state(data, method, 0)
    assert st["position"].shape == s0["position"].shape
    np.testing.assert_array_equal(st["position"], s0["position"])
    assert rel_l2(st["rest_density"], s0["rest_density"]) <= 1e-6
    for s in range(3):
        o.set_state(sph_fixture_state(data, method, s))
        o.step(1)
        assert judge_sph_step(method, o.get_state(), sph_fixture_state(data, method, s + 1)) == [], s


# ------------------------------------------------------------ frame shading
def _shade_fixture():
    return np.load(GOLDEN / "ref_shade.npz")


def test_default_camera_matches_reference_camera():
    """aq_draw_command_default against the reference's Camera + glm::lookAt /
    glm::perspective compiled from its own sources (bit for bit)."""
    import aquarius_b200 as aq
    from oracle_binding import RenderOracle
    g = _shade_fixture()
    for (w, h, size), v, p, e in zip(g["windows"], g["cam_view"], g["cam_projection"], g["cam_eye"]):
        for dc in (aq.draw_command_default(int(w), int(h), float(size), 32),
                   RenderOracle.draw_command_default(int(w), int(h), float(size), 32)):
            np.testing.assert_array_equal(np.array(dc.view, np.float32).view(np.uint32), v.view(np.uint32))
            np.testing.assert_array_equal(np.array(dc.projection, np.float32).view(np.uint32), p.view(np.uint32))
            np.testing.assert_array_equal(np.array(dc.camera_position, np.float32).view(np.uint32), e.view(np.uint32))


def test_shading_matches_reference_shaders():
    """The oracle's shading (FluidMeshRenderer_fs, RayTraceEnvironment,
    Container_face_fs restated in render_oracle.c) against the reference's own
    GLSL compiled as C++ (oracle/shade_harness.cpp), bit for bit, in every mesh
    mode and environment."""
    from oracle_binding import RenderOracle
    g = _shade_fixture()
    o = RenderOracle(sky=g["sky"], logo=g["logo"])
    dc = RenderOracle.draw_command_default(320, 160, 10.0, 32)
    for row, want in zip(g["mesh_in"], g["mesh_out"]):
        dc.environment_mode, dc.render_mode = int(row[0]), int(row[1])
        got = o.shade_mesh(dc, row[2:5], row[5:8], row[8:12])
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=str(row))
    for row, want in zip(g["trace_in"], g["trace_out"]):
        dc.environment_mode = int(row[0])
        got = o.trace(dc, row[1:4], row[4:7])
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=str(row))
    cam = np.array(dc.camera_position, np.float32)
    for row, want in zip(g["container_in"], g["container_out"]):
        dc.environment_mode = int(row[0])
        d = (row[1:4] - cam).astype(np.float32)
        dd = np.float32(np.float32(d[0] * d[0] + d[1] * d[1]) + np.float32(d[2] * d[2]))
        d = (d * np.float32(np.float32(1.0) / np.sqrt(dd))).astype(np.float32)  # GLSL normalize
        got = o.trace(dc, cam, d)
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32), err_msg=str(row))
