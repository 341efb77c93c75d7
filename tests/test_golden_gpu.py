"""The CUDA library against the committed fixtures recorded from the
reference's own kernels (no reference build needed at test time)."""
import pytest

from golden_check import judge, load, replay, replay_special, spreads
from lib_checker import LibChecker

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scene,steps", [("cfg1_16", 2), ("aniso", 1), ("multi_16", 1)])
def test_library_against_reference_fixtures(scene, steps):
    data = load(scene)
    if data is None:
        pytest.skip("fixture missing")
    directional = []
    res = replay(data, LibChecker, steps, directional=directional)
    assert judge(res, spreads().get(scene, {})) == []
    for (s, k, f, kind, v) in res:
        if kind == "int_mismatch" and not (k == 7 and f == "has_velocity"):
            assert v == 0, (s, k, f)
    assert all(v == 0 for v in directional)


def test_library_against_race_free_reference_settings():
    res = replay_special(LibChecker)
    if res is None:
        pytest.skip("fixture missing")
    for name, f, kind, v, lim in res:
        assert v <= lim, (name, f, kind, v)
