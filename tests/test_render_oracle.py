"""CPU checks of the headless-frame oracle (oracle/render_oracle.c) and of the
library's host-side camera (aq_draw_command_default), no GPU needed.

Known answers restated from the reference's shaders and GL's rules: the
default camera of main.cu, RayTraceEnvironment.glsl's chess board and sky
branches, point-sprite coverage, and a full frame of a CPU-made scene in
every render and environment mode.
"""
import math

import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi
from oracle_binding import Oracle, RenderOracle
from scenes import SCENES


def test_default_camera_library_equals_oracle():
    for w, h, size, sy in [(1728, 864, 10.0, 128), (320, 160, 10.0, 32), (97, 31, 3.5, 20)]:
        a = aq.draw_command_default(w, h, size, sy)
        b = RenderOracle.draw_command_default(w, h, size, sy)
        assert bytes(a) == bytes(b)


def test_default_camera_geometry():
    """Camera(center) (camera.h:65-93): 18 units from the centre at pitch 30
    on the -z side, looking at the centre; glm::perspective with fovy = 45 taken
    as radians."""
    dc = aq.draw_command_default(1728, 864, 10.0, 128)
    eye = np.array(dc.camera_position)
    np.testing.assert_allclose(eye, [5.0, 5.0 + 9.0, 5.0 - 18.0 * math.cos(math.radians(30))], rtol=1e-6)
    V = np.array(dc.view, np.float64).reshape(4, 4).T
    c = V @ np.array([5.0, 5.0, 5.0, 1.0])
    np.testing.assert_allclose(c[:3], [0.0, 0.0, -18.0], atol=1e-5)  # the centre straight ahead
    P = np.array(dc.projection, np.float64).reshape(4, 4).T
    assert P[1, 1] == pytest.approx(1.0 / math.tan(22.5), rel=1e-6)
    assert P[0, 0] == pytest.approx(P[1, 1] / 2.0, rel=1e-6)
    assert dc.point_radius == pytest.approx(10.0 / 128)
    assert dc.cornell_box_size == 40.0 and tuple(dc.light_position) == (5.0, 15.0, 5.0)


def _dc(w=160, h=80):
    return RenderOracle.draw_command_default(w, h, 10.0, 32)


def test_trace_sky_and_chess_board():
    """RayTraceEnvironment.glsl:155-170: a ray down into the container hits
    the chess board (cells of 1 unit, 0.5 / 0.8 grey); a ray up samples the
    cube map."""
    sky = np.zeros((6, 4, 4, 3), np.uint8)
    for f in range(6):
        sky[f] = 40 * (f + 1)
    o = RenderOracle(sky=sky)
    dc = _dc()
    c = o.trace(dc, [0.5, 2.0, 0.5], [0.0, -1.0, 0.0])  # cell (100, 100): even
    np.testing.assert_array_equal(c, [0.5, 0.5, 0.5, 1.0])
    c = o.trace(dc, [1.5, 2.0, 0.5], [0.0, -1.0, 0.0])  # cell (101, 100): odd
    np.testing.assert_allclose(c, [0.8, 0.8, 0.8, 1.0])
    c = o.trace(dc, [0.5, 2.0, 0.5], [0.0, 1.0, 0.0])  # +y face
    np.testing.assert_allclose(c[:3], 120 / 255.0, rtol=1e-6)
    c = o.trace(dc, [20.0, 2.0, 0.5], [0.0, -1.0, 0.0])  # outside the container: the sky (-y face)
    np.testing.assert_allclose(c[:3], 160 / 255.0, rtol=1e-6)


def test_trace_chess_board_mode_lighting():
    o = RenderOracle()
    dc = _dc()
    dc.environment_mode = _abi.ENV_CHESS_BOARD
    c = o.trace(dc, [5.5, 3.0, 5.5], [0.0, -1.0, 0.0])
    # hit (5.5, 0, 5.5): cell (105, 105) even -> 0.5; light (5, 15, 5)
    tl = np.array([5.0, 15.0, 5.0]) - np.array([5.5, 0.0, 5.5])
    shade = 0.1 + 0.5 * tl[1] / np.linalg.norm(tl)
    np.testing.assert_allclose(c, [0.5 * shade] * 3 + [shade], rtol=1e-5)
    c = o.trace(dc, [5.5, 3.0, 5.5], [0.0, 1.0, 0.0])
    np.testing.assert_array_equal(c, [0.0, 0.0, 0.0, 1.0])


def test_trace_cornell_box():
    o = RenderOracle()
    dc = _dc()
    dc.environment_mode = _abi.ENV_CORNELL_BOX
    # box (-15, 0, -15) .. (25, 40, 25); a ray along +x from the centre hits the x = 25 wall
    c = o.trace(dc, [5.0, 5.0, 5.0], [1.0, 0.0, 0.0])
    tl = np.array([5.0, 15.0, 5.0]) - np.array([25.0, 5.0, 5.0])
    shade = 0.1 + 0.5 * max(0.0, np.dot([-1.0, 0.0, 0.0], tl / np.linalg.norm(tl)))
    np.testing.assert_allclose(c, [0.8 * shade] * 3 + [1.0], rtol=1e-5)


def test_single_point_sprite_coverage():
    """One point at the centre of view: its phase thickness covers a disc of
    the size gl_PointSize gives (PointSprites_points_vs.glsl:30-32)."""
    dc = _dc(200, 100)
    dc.render_mode = _abi.RENDER_MULTIPHASE_MESH
    pt = np.array([[5.0, 5.0, 5.0, 0.25, 0.5, 0.0, 0.0]], np.float32)
    _, ph = RenderOracle().frame(dc, pt, None)
    covered = ph[..., 0] > 0
    tan_half = math.tan(math.radians(45.0) / 2)
    s = (100 / 2) * dc.point_radius / (tan_half * 18.0)
    assert abs(covered.sum() - math.pi * (s / 2) ** 2) <= 2 * math.pi * s / 2 + 2
    np.testing.assert_array_equal(ph[covered][:, :2], np.tile([0.25, 0.5], (covered.sum(), 1)))
    ys, xs = np.nonzero(covered)
    assert abs(xs.mean() + 0.5 - 100) < 1.0 and abs(ys.mean() + 0.5 - 50) < 1.0


def test_none_mode_is_the_cleared_frame():
    dc = _dc()
    dc.render_mode = _abi.RENDER_NONE
    img, ph = RenderOracle(sky=np.full((6, 2, 2, 3), 200, np.uint8)).frame(dc, None, None)
    assert (img[..., :3] == 0).all() and (img[..., 3] == 255).all() and not ph.any()


@pytest.fixture(scope="module")
def cpu_scene():
    cfg = SCENES["multi_16"]()
    o = Oracle(cfg)
    o.step(2)
    st = o.get_state(["position", "fractions"])
    pts = np.concatenate([st["position"].T, st["fractions"].T], axis=1).astype(np.float32)
    mesh = o.mesh()["records"].reshape(-1, 6)
    o.close()
    return cfg, pts, mesh


@pytest.mark.parametrize("env", [0, 1, 2])
@pytest.mark.parametrize("mode", list(range(10)))
def test_every_mode_draws(cpu_scene, mode, env):
    cfg, pts, mesh = cpu_scene
    rng = np.random.default_rng(3)
    o = RenderOracle(sky=rng.integers(0, 256, (6, 8, 8, 3), dtype=np.uint8),
                     logo=rng.integers(0, 256, (8, 8, 3), dtype=np.uint8))
    dc = RenderOracle.draw_command_default(96, 48, cfg.domain_size, cfg.size_y)
    dc.render_mode, dc.environment_mode = mode, env
    img, ph = o.frame(dc, pts, mesh)
    if mode == _abi.RENDER_NONE:
        assert (img[..., :3] == 0).all()
        return
    assert len(np.unique(img.reshape(-1, 4), axis=0)) > 3
    multiphase = mode in (0, 5, 6, 7)
    assert bool(ph.any()) == multiphase
    if multiphase:  # the two phases' fractions sum to 1 per particle: thickness = coverage count
        assert np.isclose(ph.sum(), ph[..., :2].sum())


def _window(dc, p):
    """Window coordinates of world point p (float64)."""
    P = np.array(dc.projection, np.float64).reshape(4, 4).T
    V = np.array(dc.view, np.float64).reshape(4, 4).T
    c = P @ V @ np.array([p[0], p[1], p[2], 1.0])
    ndc = c[:3] / c[3]
    return np.array([(ndc[0] + 1) * dc.window_width / 2, (ndc[1] + 1) * dc.window_height / 2])


def _quad_mesh(corners, normal):
    a, b, c, d = corners
    verts = [a, b, c, a, c, d]
    return np.array([list(v) + list(normal) for v in verts], np.float32)


def test_shared_edge_leaves_no_gap():
    """A quad drawn as two triangles sharing a diagonal: every pixel whose
    centre lies inside the quad is drawn (the top-left rule gives shared-edge
    pixels to exactly one triangle, none to neither)."""
    dc = _dc(400, 200)
    dc.render_mode = _abi.RENDER_FLAT_MESH
    corners = [(3.0, 6.0, 5.0), (7.0, 6.0, 5.0), (7.0, 9.0, 5.0), (3.0, 9.0, 5.0)]
    img, _ = RenderOracle().frame(dc, None, _quad_mesh(corners, (0.0, 0.0, -1.0)))
    bg, _ = RenderOracle().frame(dc, None, None)
    drawn = (img != bg).any(-1)
    w = np.array([_window(dc, c) for c in corners])
    ys, xs = np.mgrid[0:dc.window_height, 0:dc.window_width]
    px, py = xs + 0.5, ys + 0.5
    inside = np.ones_like(drawn)
    for k in range(4):  # a convex quad: inside every edge by a margin of 0.05 px
        a, b = w[k], w[(k + 1) % 4]
        e = (b[0] - a[0]) * (py - a[1]) - (b[1] - a[1]) * (px - a[0])
        sgn = np.sign((w[(k + 2) % 4][1] - a[1]) * (b[0] - a[0]) - (w[(k + 2) % 4][0] - a[0]) * (b[1] - a[1]))
        inside &= sgn * e > 0.05 * np.hypot(*(b - a))
    assert inside.sum() > 500
    assert drawn[inside].all(), int((~drawn[inside]).sum())


def test_triangle_through_the_near_plane_is_dropped():
    """A triangle with a vertex behind the eye is dropped whole (no
    clipping), as the frame rules say."""
    dc = _dc(160, 80)
    dc.render_mode = _abi.RENDER_FLAT_MESH
    eye = np.array(dc.camera_position, np.float64)
    behind = eye + (eye - np.array([5.0, 5.0, 5.0])) * 0.5
    tri = np.array([list(behind) + [0, 1, 0], [2.0, 5.0, 5.0, 0, 1, 0], [8.0, 5.0, 5.0, 0, 1, 0]], np.float32)
    img, _ = RenderOracle().frame(dc, None, tri)
    bg, _ = RenderOracle().frame(dc, None, None)
    np.testing.assert_array_equal(img, bg)
    tri[0, :3] = [5.0, 8.0, 5.0]  # the same triangle in front of the camera is drawn
    img2, _ = RenderOracle().frame(dc, None, tri)
    assert (img2 != bg).any()
