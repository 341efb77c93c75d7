"""C-ABI surface checks that need no GPU: the library loads, exports every
entry point include/aquarius_b200.h declares, and the host-only calls work."""
import ctypes as ct
import pathlib
import re

import pytest

from aquarius_b200 import _abi

ROOT = pathlib.Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "aquarius_b200.h"


def declared_functions(path=HEADER):
    text = path.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(aq_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["aq_config_default", "aq_fluid_create", "aq_fluid_step", "aq_fluid_destroy",
                 "aq_fluid_download_state", "aq_fluid_upload_state", "aq_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol(built_library):
    lib = ct.CDLL(str(built_library))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert missing == []


def test_struct_sizes_match_c(built_library):
    # offsets the C side relies on: aq_config ends with an 8-byte pointer
    assert ct.sizeof(_abi.Volume) == 4 * 12
    assert _abi.Config.stream.offset % 8 == 0
    assert ct.sizeof(_abi.HostState) == 8 * 3 + 8 * 17
    assert ct.sizeof(_abi.MeshInfo) == 4 * 9


def test_config_default_matches_reference(built_library):
    import aquarius_b200 as aq
    lib = aq.load_library()
    c = _abi.Config()
    assert lib.aq_config_default(ct.byref(c)) == 0
    py = _abi.default_config_values(_abi.Config())
    assert bytes(c) == bytes(py)
    assert (c.size_x, c.pressure_iterations, c.diffusion_iterations) == (50, 100, 100)
    assert abs(c.timestep - 0.033) < 1e-7 and abs(c.flip_coeff - 0.95) < 1e-7
    assert list(c.gravity) == pytest.approx([0, -9.8, 0])
    assert c.volume_count == 2 and c.volumes[0].shape == _abi.SHAPE_SQUARE


@pytest.mark.parametrize("field,value,ok", [
    ("size_x", 3, False), ("size_x", 4, True), ("phase_count", 5, False), ("phase_count", 4, True),
    ("pressure_iterations", -1, False), ("timestep", -0.1, False), ("domain_size", 0.0, False),
])
def test_config_validation(built_library, field, value, ok):
    import aquarius_b200 as aq
    lib = aq.load_library()
    c = _abi.make_config((16, 16, 16))
    setattr(c, field, value)
    st = lib.aq_config_validate(ct.byref(c))
    assert (st == 0) == ok
    if not ok:
        assert st == 1  # AQ_ERR_INVALID_CONFIG
        assert lib.aq_last_error()


def test_phase_out_of_range_rejected(built_library):
    import aquarius_b200 as aq
    lib = aq.load_library()
    c = _abi.make_config((16, 16, 16), [dict(shape="box", phase=4)])
    assert lib.aq_config_validate(ct.byref(c)) == 1


def test_residual_mode_validation(built_library):
    import aquarius_b200 as aq
    lib = aq.load_library()
    c = _abi.make_config((16, 16, 16), solve_mode=_abi.SOLVE_RESIDUAL, check_interval=0)
    assert lib.aq_config_validate(ct.byref(c)) == 1
    c = _abi.make_config((16, 16, 16), solve_mode=_abi.SOLVE_RESIDUAL, check_interval=40, max_iterations=2000)
    assert lib.aq_config_validate(ct.byref(c)) == 0


def test_python_config_roundtrip():
    import aquarius_b200 as aq
    fc = aq.FluidConfig()
    c = fc.to_c()
    assert bytes(c) == bytes(_abi.default_config_values(_abi.Config()))
    fc.FLIP.sizeX = 64
    fc.solveMode = "residual"
    c = fc.to_c()
    assert c.size_x == 64 and c.solve_mode == _abi.SOLVE_RESIDUAL


def test_null_arguments_are_rejected(built_library):
    import aquarius_b200 as aq
    lib = aq.load_library()
    assert lib.aq_fluid_create(None, None) == 2  # AQ_ERR_INVALID_ARGUMENT
    assert lib.aq_fluid_step(None, 1) == 2
    assert lib.aq_abi_version() == 1


def test_create_without_gpu_fails_cleanly(built_library):
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    import aquarius_b200 as aq
    with pytest.raises(aq.AquariusError) as e:
        aq.Fluid(aq.FluidConfig())
    assert e.value.status == 7  # AQ_ERR_NO_DEVICE


def test_sph_config_default_matches_reference(built_library):
    import aquarius_b200 as aq
    lib = aq.load_library()
    for method in (_abi.SPH_PBF, _abi.SPH_PCISPH):
        c = _abi.SphConfig()
        assert lib.aq_sph_config_default(method, ct.byref(c)) == 0
        assert bytes(c) == bytes(_abi.sph_config(method))
    assert ct.sizeof(_abi.SphState) == 8 + 8 + 8 * 10
    assert ct.sizeof(_abi.SphInfo) == 4 * 7
