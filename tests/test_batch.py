"""Scene batches, host side (no GPU): the seeded scene set and the checks
aq_batch_create makes before it touches a device."""
import ctypes as ct

import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi
from aquarius_b200.scenes import BATCH_SIZES, batch_configs
from conftest import gpu_available


def test_scene_set_is_seeded_and_in_range():
    a = batch_configs(64, seed=7)
    b = batch_configs(64, seed=7)
    c = batch_configs(64, seed=8)
    key = lambda cs: [(x.size_x, x.size_y, x.size_z, x.volume_count, x.volumes[0].box_max[1]) for x in cs]
    assert key(a) == key(b)
    assert key(a) != key(c)
    sizes = set()
    for cfg in a:
        for s in (cfg.size_x, cfg.size_y, cfg.size_z):
            assert s in BATCH_SIZES
            sizes.add(s)
        assert cfg.size_z % 4 == 0
        assert 2 <= cfg.volume_count <= 3
        assert 0.1 <= cfg.volumes[0].box_max[1] <= 0.4
        for v in cfg.volumes[1:cfg.volume_count]:
            assert v.shape == _abi.SHAPE_SPHERE
            assert 0.08 <= v.ball_radius <= 0.2
            assert 0.0 <= min(v.ball_center) and max(v.ball_center) <= 1.0
        assert len({v.phase for v in cfg.volumes[:cfg.volume_count]}) == 1
    assert sizes == set(BATCH_SIZES)  # anisotropic and uneven


def _create(cfgs):
    lib = aq.load_library()
    arr = (_abi.Config * len(cfgs))(*cfgs)
    h = ct.c_void_p()
    st = lib.aq_batch_create(arr, len(cfgs), ct.byref(h))
    if h.value:
        lib.aq_batch_destroy(h)
    return st, (lib.aq_last_error() or b"").decode()


@pytest.mark.parametrize("mutate,needle", [
    (lambda cs: setattr(cs[1], "size_z", 30), "size_z % 4"),
    (lambda cs: setattr(cs[1], "pressure_iterations", 7), "share the pressure solver"),
    (lambda cs: [setattr(c, "check_interval", 7) for c in cs], "even check_interval"),
    (lambda cs: setattr(cs[1].volumes[1], "phase", 1), "single-phase"),
    (lambda cs: setattr(cs[1], "size_x", 2), "sizes must be >= 4"),
])
def test_create_rejects_unbatchable_configs(built_library, mutate, needle):
    cfgs = batch_configs(3, seed=1, sizes=(16, 24))
    mutate(cfgs)
    st, msg = _create(cfgs)
    assert _abi.STATUS_NAMES[st] == "AQ_ERR_INVALID_CONFIG"
    assert needle in msg


def test_create_rejects_empty_batch(built_library):
    lib = aq.load_library()
    h = ct.c_void_p()
    assert _abi.STATUS_NAMES[lib.aq_batch_create(None, 0, ct.byref(h))] == "AQ_ERR_INVALID_ARGUMENT"


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_create_without_device_fails_loudly(built_library):
    st, msg = _create(batch_configs(3, seed=1, sizes=(16, 24)))
    assert _abi.STATUS_NAMES[st] == "AQ_ERR_NO_DEVICE"


def test_learned_mode_validation(built_library):
    from aquarius_b200.scenes import batch_configs as bc
    lib = aq.load_library()
    ok = _abi.make_config((16, 16, 16), None, pressure_init=_abi.PRESSURE_LEARNED, solve_mode=_abi.SOLVE_RESIDUAL)
    assert lib.aq_config_validate(ct.byref(ok)) == 0
    bad = _abi.make_config((18, 16, 16), None, pressure_init=_abi.PRESSURE_LEARNED)
    assert _abi.STATUS_NAMES[lib.aq_config_validate(ct.byref(bad))] == "AQ_ERR_INVALID_CONFIG"
    few = _abi.make_config((16, 16, 16), None, pressure_init=_abi.PRESSURE_LEARNED, solve_mode=_abi.SOLVE_FIXED,
                           pressure_iterations=10)
    assert _abi.STATUS_NAMES[lib.aq_config_validate(ct.byref(few))] == "AQ_ERR_INVALID_CONFIG"
    cfgs = bc(2, seed=1, sizes=(16,), pressure_init=_abi.PRESSURE_LEARNED)
    st, msg = _create(cfgs)
    assert _abi.STATUS_NAMES[st] == "AQ_ERR_INVALID_CONFIG" and "learned" in msg
