"""Failure reporting without a GPU fault (the reference prints and exits on a
CUDA error, Common/GpuCommons.h:118-142, and has no check for NaN or for a
solve that stops short).

* A NaN particle velocity placed in a host-prepared upload makes the next
  step's divergence norm non-finite: aq_fluid_synchronize returns
  AQ_ERR_NONFINITE, and a clean upload clears it.
* A residual-mode solve that stops at max_iterations reports
  AQ_ERR_NOT_CONVERGED from aq_fluid_solve_stats with the achieved residual.
* A persistent solve whose grid barrier never fills (one CTA withheld by the
  test hook, a short poll limit) gives up: AQ_ERR_TIMEOUT, and the device
  keeps answering (the same fluid after an upload, and a new fluid checked
  against the oracle).
* A tcgen05 convolution whose MMAs are never issued (test hook) gives up its
  bounded mbarrier wait: nothing is written, aq_conv3_umma_status reports the
  timeout, and with the hook off the same call matches PyTorch again.
"""
import ctypes as ct

import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi
from oracle_binding import Oracle
from scenes import SCENES, rel_l2

pytestmark = pytest.mark.gpu


def _status(exc_info):
    return exc_info.value.status


def test_nan_velocity_in_upload_reports_nonfinite():
    cfg = SCENES["cfg2_32"]()
    f = aq.Fluid(cfg)
    f.step(2)
    f.synchronize()
    clean = f.download_state()
    bad = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in clean.items()}
    bad["velocity_p"][1, f.particleCount // 2] = np.nan
    f.upload_state(bad)
    f.step(1)
    with pytest.raises(aq.AquariusError) as e:
        f.synchronize()
    assert _status(e) == _abi.AQ_ERR_NONFINITE
    assert f.solve_stats()["status"] == "AQ_ERR_NONFINITE"
    with pytest.raises(aq.AquariusError) as e:  # sticky
        f.synchronize()
    assert _status(e) == _abi.AQ_ERR_NONFINITE
    f.upload_state(clean)
    f.step(1)
    f.synchronize()
    f.close()


def test_residual_cap_reports_not_converged():
    cfg = SCENES["cfg2_32"](solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=1e-12, max_iterations=40,
                            check_interval=20)
    f = aq.Fluid(cfg)
    f.step(2)
    f.synchronize()  # not converging is not an error of the step
    st = f.solve_stats()
    assert st["status"] == "AQ_ERR_NOT_CONVERGED"
    assert not st["converged"] and st["iterations"] == 40 and 0 < st["rel_residual"] < 1
    f.close()
    cfg = SCENES["cfg2_32"](solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=0.5, max_iterations=2000,
                            check_interval=20)
    f = aq.Fluid(cfg)
    f.step(2)
    st = f.solve_stats()
    assert st["status"] == "AQ_OK" and st["converged"]
    f.close()


@pytest.mark.parametrize("mode", [_abi.SOLVE_FIXED, _abi.SOLVE_RESIDUAL])
def test_persistent_barrier_timeout_leaves_device_usable(mode):
    cfg = SCENES["cfg2_32"](solve_mode=mode, rel_residual=1e-4, max_iterations=400, check_interval=20)
    f = aq.Fluid(cfg)
    f.step(1)
    f.synchronize()
    clean = f.download_state()
    f.set_jacobi_plan(1, 1, 1)  # the whole solve in one cooperative launch
    f.test_barrier_timeout(withhold_cta=1, spin_limit=1 << 14)
    f.step(1)
    with pytest.raises(aq.AquariusError) as e:
        f.synchronize()
    assert _status(e) == _abi.AQ_ERR_TIMEOUT
    # the same fluid, hook off, from a clean upload
    f.test_barrier_timeout(-1, 0)
    f.upload_state(clean)
    f.step(1)
    f.synchronize()
    f.close()
    # a new fluid steps as the oracle does
    cfg1 = SCENES["cfg1_16"]()
    g = aq.Fluid(cfg1)
    o = Oracle(cfg1)
    g.step(1)
    o.step(1)
    a, b = g.download_state(["pressure", "content"]), o.get_state(["pressure", "content"])
    np.testing.assert_array_equal(a["content"], b["content"])
    assert rel_l2(a["pressure"], b["pressure"]) <= 1e-5
    g.close()
    o.close()


def test_umma_wait_timeout_writes_nothing_and_recovers():
    import torch
    lib = aq.load_library()
    P, I = ct.c_void_p, ct.c_int32
    lib.aq_conv3_forward.restype = ct.c_int
    lib.aq_conv3_forward.argtypes = [I, I, I, P, P, P, P, I, I, I, P]
    lib.aq_conv3_set_tiled.argtypes = [I]
    lib.aq_conv3_umma_status.restype = ct.c_int
    lib.aq_conv3_umma_status.argtypes = [ct.POINTER(I)]
    lib.aq_conv3_test_wait_timeout.restype = ct.c_int
    lib.aq_conv3_test_wait_timeout.argtypes = [I, ct.c_uint64]
    shape, cin, cout = (5, 6, 7), 16, 16
    V = shape[0] * shape[1] * shape[2]
    g = torch.Generator(device="cuda").manual_seed(11)
    x = torch.randn(V, cin, device="cuda", generator=g).to(torch.bfloat16)
    w = (torch.randn(27, cout, cin, device="cuda", generator=g) * 0.1).to(torch.bfloat16)
    b = torch.randn(cout, device="cuda", generator=g)
    sentinel = torch.full((V, cout), 7.0, device="cuda", dtype=torch.bfloat16)
    out = sentinel.clone()
    status = ct.c_int32(-1)
    assert lib.aq_conv3_set_tiled(2) == 0
    assert lib.aq_conv3_test_wait_timeout(1, 20_000_000) == 0  # 20 ms wait
    try:
        assert lib.aq_conv3_forward(cin, cout, 0, x.data_ptr(), w.data_ptr(), b.data_ptr(), out.data_ptr(),
                                    *shape, None) == 0
        torch.cuda.synchronize()
        assert lib.aq_conv3_umma_status(ct.byref(status)) == 0
        assert status.value != 0
        assert torch.equal(out, sentinel)
    finally:
        assert lib.aq_conv3_test_wait_timeout(0, 0) == 0
    assert lib.aq_conv3_umma_status(ct.byref(status)) == 0 and status.value == 0
    assert lib.aq_conv3_forward(cin, cout, 0, x.data_ptr(), w.data_ptr(), b.data_ptr(), out.data_ptr(),
                                *shape, None) == 0
    torch.cuda.synchronize()
    ref = torch.nn.functional.conv3d(
        x.float().reshape(*shape, cin).permute(3, 0, 1, 2)[None],
        w.float().reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2), b, padding=1)
    got = out.float().reshape(*shape, cout).permute(3, 0, 1, 2)[None]
    assert float((got - ref).norm() / ref.norm()) < 8e-3
    assert lib.aq_conv3_umma_status(ct.byref(status)) == 0 and status.value == 0
