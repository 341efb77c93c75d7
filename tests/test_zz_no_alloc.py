"""aq_jacobi_sweeps_noalloc: the entry point for callers that cannot allocate
device memory while they run the solver (a fixed pool handed over by a host
application, a memory-budgeted frame loop, a plugin that must not touch its
host's allocator).  Its scratch is a fixed device array inside the library.

Checked through the C ABI against the fluid's own pressure stage
(aq_fluid_run_stage, AQ_STAGE_PRESSURE) on the same system, twice in a row,
since the scratch array keeps the previous call's contents.  This file is
collected last so a failure here leaves every other test already run.
"""
import ctypes as ct

import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi
from scenes import SCENES, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative L2, as the other float parity tests


def _lib():
    lib = aq.load_library()
    lib.aq_jacobi_sweeps_noalloc.restype = ct.c_int
    lib.aq_jacobi_sweeps_noalloc.argtypes = [ct.c_int32, ct.c_int32, ct.c_int32, ct.c_void_p, ct.c_void_p,
                                             ct.c_void_p, ct.c_int32, ct.c_void_p]
    lib.aq_jacobi_noalloc_max_cells.restype = ct.c_int32
    return lib


def _system(cfg):
    """A pressure system from a few real steps: cell types, rhs and the
    initial guess, plus the fluid's own solve of it."""
    f = aq.Fluid(cfg)
    f.step(3)
    for k in range(1, 5):
        f.run_stage(k)
    st = f.download_state(["content", "divergence", "density", "pressure"])
    sx, sy, sz = cfg.size_x, cfg.size_y, cfg.size_z
    fluid = st["content"].reshape(sx + 1, sy + 1, sz + 1)[:sx, :sy, :sz].ravel() == 1
    cell_type = fluid.astype(np.int8)
    rhs = np.where(fluid, (-st["divergence"]) * st["density"], np.float32(0)).astype(np.float32)
    p0 = st["pressure"].copy()
    f.run_stage(_abi.STAGE_PRESSURE)
    p_ref = f.download_state(["pressure"])["pressure"]
    f.close()
    return cell_type, rhs, p0, p_ref


def test_noalloc_matches_pressure_stage_twice():
    import torch
    cfg = SCENES["cfg2_32"](pressure_iterations=37)
    cell_type, rhs, p0, p_ref = _system(cfg)
    lib = _lib()
    dev = torch.device("cuda", 0)
    t_type = torch.from_numpy(cell_type).to(dev)
    t_rhs = torch.from_numpy(rhs).to(dev)
    for call in range(2):
        t_p = torch.from_numpy(p0.copy()).to(dev)
        torch.cuda.synchronize()
        st = lib.aq_jacobi_sweeps_noalloc(cfg.size_x, cfg.size_y, cfg.size_z, t_type.data_ptr(), t_rhs.data_ptr(),
                                          t_p.data_ptr(), 37, None)
        assert st == 0, lib.aq_last_error()
        torch.cuda.synchronize()
        got = t_p.cpu().numpy()
        e = rel_l2(got, p_ref)
        assert e <= TOL, (call, e)


def test_noalloc_rejects_grids_over_its_limit():
    lib = _lib()
    limit = lib.aq_jacobi_noalloc_max_cells()
    assert limit == 64 * 64 * 64
    st = lib.aq_jacobi_sweeps_noalloc(65, 64, 64, 16, 16, 16, 1, None)
    assert st == 2  # AQ_ERR_INVALID_ARGUMENT
    assert b"exceeds" in lib.aq_last_error()
