"""Headless frame through the C ABI (aq_renderer_draw / aq_fluid_draw).

The library walks per-tile lists of primitives pixel by pixel; the oracle
(oracle/render_oracle.c) draws GL-style, primitive by primitive.  Both follow
the same fixed-function rules, so the images are equal byte for byte except
where CUDA's expf and glibc's expf round differently (the attenuation of the
multiphase modes); there at most 1 pixel in 10^4 may differ, by at most 2/255.
The phase-thickness texture (additions only) is bit for bit equal.
"""
import numpy as np
import pytest
import torch

import aquarius_b200 as aq
from aquarius_b200 import _abi
from oracle_binding import RenderOracle
from scenes import SCENES, ball_drop

pytestmark = pytest.mark.gpu

MODES = list(range(10))
ENVS = [_abi.ENV_SKYBOX, _abi.ENV_CORNELL_BOX, _abi.ENV_CHESS_BOARD]


def _textures(seed=7, face=16, logo=(12, 20)):
    rng = np.random.default_rng(seed)
    sky = rng.integers(0, 256, (6, face, face, 3), dtype=np.uint8)
    lg = rng.integers(0, 256, (logo[0], logo[1], 3), dtype=np.uint8)
    return sky, lg


def _scene(name="multi_16", steps=3):
    cfg = SCENES[name]()
    cfg.device = 0
    f = aq.Fluid(cfg)
    f.step(steps)
    return cfg, f


def _vbos(f):
    recs = f.download_mesh()
    mesh = np.ascontiguousarray(recs.reshape(-1, 6))
    pts = torch.empty(f.particleCount * 7, dtype=torch.float32, device="cuda")
    f.points_vbo_into(pts.data_ptr())
    torch.cuda.synchronize()
    return pts.cpu().numpy().reshape(-1, 7), mesh


def _draw(r, dc, points, mesh):
    h, w = dc.window_height, dc.window_width
    out = torch.zeros(h * w * 4, dtype=torch.uint8, device="cuda")
    tp = torch.from_numpy(points).cuda() if points is not None and len(points) else None
    tm = torch.from_numpy(mesh).cuda() if mesh is not None and len(mesh) else None
    r.draw(dc, 0 if tp is None else tp.data_ptr(), 0 if tp is None else points.shape[0],
           0 if tm is None else tm.data_ptr(), 0 if tm is None else mesh.shape[0], out.data_ptr())
    r.synchronize()
    return out.cpu().numpy().reshape(h, w, 4), r.phase_thickness()


def _compare(got, want, where=""):
    diff = np.abs(got.astype(np.int16) - want.astype(np.int16)).max(axis=-1)
    bad = np.count_nonzero(diff)
    assert diff.max() <= 2, (where, int(diff.max()), np.argwhere(diff > 2)[:5])
    assert bad <= max(1, diff.size // 10000), (where, bad)


@pytest.fixture(scope="module")
def small():
    cfg, f = _scene()
    pts, mesh = _vbos(f)
    sky, logo = _textures()
    r = aq.Renderer(0)
    r.set_skybox(sky)
    r.set_logo(logo)
    yield dict(cfg=cfg, f=f, pts=pts, mesh=mesh, sky=sky, logo=logo, r=r, o=RenderOracle(sky=sky, logo=logo))
    r.close()
    f.close()


@pytest.mark.parametrize("env", ENVS)
@pytest.mark.parametrize("mode", MODES)
def test_frame_matches_oracle(small, mode, env):
    cfg = small["cfg"]
    dc = aq.draw_command_default(320, 160, cfg.domain_size, cfg.size_y)
    dc.render_mode = mode
    dc.environment_mode = env
    if mode == _abi.RENDER_PARTICLES:
        dc.point_radius = dc.point_radius / 2.0  # renderRadius = cellPhysicalSize / 8^(1/3)
    got, gph = _draw(small["r"], dc, small["pts"], small["mesh"])
    want, wph = small["o"].frame(dc, small["pts"], small["mesh"])
    np.testing.assert_array_equal(gph, wph)
    _compare(got, want, (mode, env))
    if mode != _abi.RENDER_NONE:
        assert len(np.unique(got.reshape(-1, 4), axis=0)) > 3, "a blank frame"


def test_fluid_draw_equals_explicit_vbos(small):
    cfg, f = small["cfg"], small["f"]
    dc = aq.draw_command_default(256, 128, cfg.domain_size, cfg.size_y)
    f.draw(dc, small["r"])
    a = small["r"].image()
    b, _ = _draw(small["r"], dc, small["pts"], small["mesh"])
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("wh", [(1, 1), (17, 33), (333, 197), (64, 64)])
def test_ragged_windows(small, wh):
    cfg = small["cfg"]
    dc = aq.draw_command_default(wh[0], wh[1], cfg.domain_size, cfg.size_y)
    got, gph = _draw(small["r"], dc, small["pts"], small["mesh"])
    want, wph = small["o"].frame(dc, small["pts"], small["mesh"])
    np.testing.assert_array_equal(gph, wph)
    _compare(got, want, wh)


def test_empty_inputs_and_none_mode(small):
    cfg = small["cfg"]
    dc = aq.draw_command_default(96, 48, cfg.domain_size, cfg.size_y)
    for mode in (_abi.RENDER_MULTIPHASE_MESH, _abi.RENDER_PARTICLES):
        dc.render_mode = mode
        got, gph = _draw(small["r"], dc, None, None)
        want, _ = small["o"].frame(dc, None, None)
        _compare(got, want, mode)
        assert not gph.any()
    dc.render_mode = _abi.RENDER_NONE
    got, _ = _draw(small["r"], dc, small["pts"], small["mesh"])
    assert (got[..., :3] == 0).all() and (got[..., 3] == 255).all()


def test_camera_inside_the_fluid(small):
    """Triangles crossing the near plane are dropped whole on both sides."""
    cfg = small["cfg"]
    dc = aq.draw_command_default(200, 100, cfg.domain_size, cfg.size_y)
    # move the eye down to the pool surface, looking along +z
    V = np.array(dc.view, np.float32).reshape(4, 4).T
    V[:3, 3] = 0
    eye = np.array([cfg.domain_size * 0.5, cfg.domain_size * 0.3, cfg.domain_size * 0.05], np.float32)
    V[:3, 3] = -(V[:3, :3] @ eye)
    dc.view[:] = V.T.reshape(-1).tolist()
    dc.camera_position[:] = eye.tolist()
    got, _ = _draw(small["r"], dc, small["pts"], small["mesh"])
    want, _ = small["o"].frame(dc, small["pts"], small["mesh"])
    _compare(got, want, "inside")


def test_no_textures_sample_black(small):
    cfg = small["cfg"]
    r = aq.Renderer(0)
    o = RenderOracle()
    dc = aq.draw_command_default(128, 64, cfg.domain_size, cfg.size_y)
    got, _ = _draw(r, dc, small["pts"], small["mesh"])
    want, _ = o.frame(dc, small["pts"], small["mesh"])
    _compare(got, want, "no textures")
    r.close()


def test_full_size_frame_matches_oracle():
    """The bench frame: 128^3 ball drop (5.2M particles) at 1728x864."""
    cfg = ball_drop((128, 128, 128), pool=0.3, center=(0.5, 0.7, 0.5), radius=0.12, dt=0.005)
    cfg.device = 0
    f = aq.Fluid(cfg)
    f.step(2)
    pts, mesh = _vbos(f)
    sky, logo = _textures(face=64)
    r = aq.Renderer(0)
    r.set_skybox(sky)
    dc = aq.draw_command_default(1728, 864, cfg.domain_size, cfg.size_y)
    got, gph = _draw(r, dc, pts, mesh)
    want, wph = RenderOracle(sky=sky).frame(dc, pts, mesh)
    np.testing.assert_array_equal(gph, wph)
    _compare(got, want, "full")
    assert gph[..., 0].sum() > 0
    r.close()
    f.close()
