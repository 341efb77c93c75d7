"""aq_jacobi_sweeps_noalloc: the entry point for callers that cannot allocate
device memory while they run the solver (a fixed pool handed over by a host
application, a memory-budgeted frame loop, a plugin that must not touch its
host's allocator).  Its scratch is a fixed device array inside the library.

Checked through the C ABI against the fluid's own pressure stage
(aq_fluid_run_stage, AQ_STAGE_PRESSURE) on the same system.  The sweeps are
the same kernels in the same order, so the result must be bit for bit the
stage's.  The scratch array keeps the previous call's contents, so the calls
run back to back on different systems (grid sizes, fluid cells, right-hand
sides, and a z extent that is not a multiple of 4, which takes the tiled
kernels), each compared with its own pressure stage.  This file is collected
last so a failure here leaves every other test already run.
"""
import ctypes as ct

import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi
from scenes import SCENES, ball_drop

pytestmark = pytest.mark.gpu


def _lib():
    lib = aq.load_library()
    lib.aq_jacobi_sweeps_noalloc.restype = ct.c_int
    lib.aq_jacobi_sweeps_noalloc.argtypes = [ct.c_int32, ct.c_int32, ct.c_int32, ct.c_void_p, ct.c_void_p,
                                             ct.c_void_p, ct.c_int32, ct.c_void_p]
    lib.aq_jacobi_noalloc_max_cells.restype = ct.c_int32
    return lib


def _system(cfg, steps=3):
    """A pressure system from a few real steps: the fluid's cell types (0 air,
    1 fluid, 2 solid), rhs and the initial guess, plus the fluid's own solve
    of it."""
    f = aq.Fluid(cfg)
    f.step(steps)
    for k in range(1, 5):
        f.run_stage(k)
    st = f.download_state(["content", "divergence", "density", "pressure"])
    sx, sy, sz = cfg.size_x, cfg.size_y, cfg.size_z
    content = st["content"].reshape(sx + 1, sy + 1, sz + 1)[:sx, :sy, :sz].ravel()
    fluid = content == 1
    cell_type = content.astype(np.int8)
    rhs = np.where(fluid, (-st["divergence"]) * st["density"], np.float32(0)).astype(np.float32)
    p0 = st["pressure"].copy()
    f.run_stage(_abi.STAGE_PRESSURE)
    p_ref = f.download_state(["pressure"])["pressure"]
    f.close()
    return (sx, sy, sz), cell_type, rhs, p0, p_ref


def _call(lib, system, sweeps):
    import torch
    (sx, sy, sz), cell_type, rhs, p0, _ = system
    dev = torch.device("cuda", 0)
    t_type = torch.from_numpy(cell_type).to(dev)
    t_rhs = torch.from_numpy(rhs).to(dev)
    t_p = torch.from_numpy(p0.copy()).to(dev)
    torch.cuda.synchronize()
    st = lib.aq_jacobi_sweeps_noalloc(sx, sy, sz, t_type.data_ptr(), t_rhs.data_ptr(), t_p.data_ptr(), sweeps, None)
    assert st == 0, lib.aq_last_error()
    torch.cuda.synchronize()
    return t_p.cpu().numpy()


def test_noalloc_matches_pressure_stage_on_consecutive_systems():
    sweeps = 37  # odd: the result is copied back from the scratch buffer
    a = _system(SCENES["cfg2_32"](pressure_iterations=sweeps))
    # another size, fluid layout and right-hand side; sz = 30 is not a
    # multiple of 4, so this call takes the tiled sweep kernels
    b = _system(ball_drop((30, 28, 30), pool=0.35, center=(0.4, 0.7, 0.6), radius=0.18,
                          pressure_iterations=sweeps), steps=4)
    assert a[1].shape != b[1].shape
    lib = _lib()
    for i, s in enumerate([a, b, a]):
        got = _call(lib, s, sweeps)
        assert np.array_equal(got, s[4]), (i, float(np.abs(got - s[4]).max()))


def test_noalloc_allocates_no_device_memory():
    import torch
    sweeps = 12
    s = _system(SCENES["cfg2_32"](pressure_iterations=sweeps))
    lib = _lib()
    got = _call(lib, s, sweeps)  # first call: the array's address lookup and module loading
    assert np.array_equal(got, s[4])
    (sx, sy, sz), cell_type, rhs, p0, _ = s
    dev = torch.device("cuda", 0)
    t_type = torch.from_numpy(cell_type).to(dev)
    t_rhs = torch.from_numpy(rhs).to(dev)
    t_p = torch.from_numpy(p0.copy()).to(dev)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(3):
        assert lib.aq_jacobi_sweeps_noalloc(sx, sy, sz, t_type.data_ptr(), t_rhs.data_ptr(), t_p.data_ptr(),
                                            sweeps, None) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0


def test_noalloc_rejects_grids_over_its_limit():
    lib = _lib()
    limit = lib.aq_jacobi_noalloc_max_cells()
    assert limit == 64 * 64 * 64
    st = lib.aq_jacobi_sweeps_noalloc(65, 64, 64, 16, 16, 16, 1, None)
    assert st == 2  # AQ_ERR_INVALID_ARGUMENT
    assert b"exceeds" in lib.aq_last_error()
