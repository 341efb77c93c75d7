"""The U-Net's hand-written BF16 convolution kernels against PyTorch's FP32
conv3d (the test oracle for these kernels): forward, data gradient (forward
on the flipped, transposed weights) and weight gradient, on odd grid sizes
(partial tiles, every boundary) and for every channel pair the network uses.
The forward runs in three variants: tcgen05 UMMA with TMEM accumulators (the
default where it fits), halo-tiled mma.sync and im2col mma.sync."""
import ctypes as ct

import numpy as np
import pytest

import aquarius_b200 as aq

pytestmark = pytest.mark.gpu

FWD_PAIRS = [(16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (48, 16), (32, 16), (64, 32), (32, 96),
             (16, 48)]
LAYER_PAIRS = [(16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (48, 16)]


def _lib():
    lib = aq.load_library()
    P, I = ct.c_void_p, ct.c_int32
    lib.aq_conv3_forward.restype = ct.c_int
    lib.aq_conv3_forward.argtypes = [I, I, I, P, P, P, P, I, I, I, P]
    lib.aq_conv3_weight_grad.restype = ct.c_int
    lib.aq_conv3_weight_grad.argtypes = [I, I, P, P, P, I, I, I, P]
    lib.aq_conv3_flip_transpose.restype = ct.c_int
    lib.aq_conv3_flip_transpose.argtypes = [I, I, P, P, P]
    lib.aq_conv3_set_tiled.restype = ct.c_int
    lib.aq_conv3_set_tiled.argtypes = [I]
    lib.aq_conv3_umma_status.restype = ct.c_int
    lib.aq_conv3_umma_status.argtypes = [ct.POINTER(I)]
    return lib


def _no_umma_timeouts(lib):
    v = ct.c_int32(-1)
    assert lib.aq_conv3_umma_status(ct.byref(v)) == 0
    assert v.value == 0, "a tcgen05 convolution gave up waiting for its MMAs"


def _torch():
    import torch
    torch.backends.cudnn.allow_tf32 = False
    torch.backends.cuda.matmul.allow_tf32 = False
    return torch


def _to_ncdhw(t, shape):
    sx, sy, sz = shape
    return t.float().reshape(sx, sy, sz, -1).permute(3, 0, 1, 2)[None]


def _w_torch(w, cin, cout):
    # w[tap][co][ci], tap = (dx+1)*9 + (dy+1)*3 + (dz+1) -> [co][ci][dx][dy][dz]
    return w.float().reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2).contiguous()


def _rel(a, b):
    return float((a - b).norm() / max(b.norm(), 1e-30))


@pytest.mark.parametrize("tiled", [2, 1, 0], ids=["umma", "tiled", "im2col"])
@pytest.mark.parametrize("cin,cout", FWD_PAIRS)
@pytest.mark.parametrize("shape", [(5, 6, 7), (12, 8, 16), (8, 12, 36)])
def test_conv3_forward_matches_torch(cin, cout, shape, tiled):
    torch = _torch()
    lib = _lib()
    assert lib.aq_conv3_set_tiled(tiled) == 0
    g = torch.Generator(device="cuda").manual_seed(cin * 100 + cout)
    V = shape[0] * shape[1] * shape[2]
    x = torch.randn(V, cin, device="cuda", generator=g).to(torch.bfloat16)
    w = (torch.randn(27, cout, cin, device="cuda", generator=g) * 0.1).to(torch.bfloat16)
    b = torch.randn(cout, device="cuda", generator=g)
    out = torch.empty(V, cout, device="cuda", dtype=torch.bfloat16)
    for relu in (0, 1):
        assert lib.aq_conv3_forward(cin, cout, relu, x.data_ptr(), w.data_ptr(), b.data_ptr(), out.data_ptr(),
                                    *shape, None) == 0
        torch.cuda.synchronize()
        ref = torch.nn.functional.conv3d(_to_ncdhw(x, shape), _w_torch(w, cin, cout), b, padding=1)
        if relu:
            ref = torch.relu(ref)
        got = _to_ncdhw(out, shape)
        assert _rel(got, ref) < 8e-3  # bf16 rounding of the output
    _no_umma_timeouts(lib)
    lib.aq_conv3_set_tiled(2)


def test_tiled_and_im2col_agree_bitwise():
    torch = _torch()
    lib = _lib()
    shape = (9, 10, 20)
    V = shape[0] * shape[1] * shape[2]
    g = torch.Generator(device="cuda").manual_seed(5)
    for cin, cout in FWD_PAIRS:
        x = torch.randn(V, cin, device="cuda", generator=g).to(torch.bfloat16)
        w = (torch.randn(27, cout, cin, device="cuda", generator=g) * 0.1).to(torch.bfloat16)
        b = torch.randn(cout, device="cuda", generator=g)
        outs = []
        for tiled in (1, 0):
            lib.aq_conv3_set_tiled(tiled)
            o = torch.empty(V, cout, device="cuda", dtype=torch.bfloat16)
            assert lib.aq_conv3_forward(cin, cout, 1, x.data_ptr(), w.data_ptr(), b.data_ptr(), o.data_ptr(),
                                        *shape, None) == 0
            outs.append(o)
        torch.cuda.synchronize()
        assert torch.equal(outs[0], outs[1]), (cin, cout)
    lib.aq_conv3_set_tiled(2)


@pytest.mark.parametrize("cin,cout", LAYER_PAIRS)
def test_conv3_gradients_match_torch(cin, cout):
    torch = _torch()
    lib = _lib()
    shape = (9, 6, 8)
    V = shape[0] * shape[1] * shape[2]
    g = torch.Generator(device="cuda").manual_seed(7 + cin + cout)
    x = torch.randn(V, cin, device="cuda", generator=g).to(torch.bfloat16)
    w = (torch.randn(27, cout, cin, device="cuda", generator=g) * 0.1).to(torch.bfloat16)
    dy = torch.randn(V, cout, device="cuda", generator=g).to(torch.bfloat16)
    # weight gradient
    dw = torch.empty(27, cout, cin, device="cuda", dtype=torch.float32)
    assert lib.aq_conv3_weight_grad(cin, cout, x.data_ptr(), dy.data_ptr(), dw.data_ptr(), *shape, None) == 0
    torch.cuda.synchronize()
    ref_dw = torch.nn.grad.conv3d_weight(_to_ncdhw(x, shape), (cout, cin, 3, 3, 3), _to_ncdhw(dy, shape), padding=1)
    assert _rel(_w_torch(dw, cin, cout), ref_dw) < 1e-5  # exact products, f32 sums in another order
    # data gradient: forward convolution of dy with the flipped, transposed weights
    wt = torch.empty(27, cin, cout, device="cuda", dtype=torch.bfloat16)
    assert lib.aq_conv3_flip_transpose(cin, cout, w.data_ptr(), wt.data_ptr(), None) == 0
    dx = torch.empty(V, cin, device="cuda", dtype=torch.bfloat16)
    assert lib.aq_conv3_forward(cout, cin, 0, dy.data_ptr(), wt.data_ptr(), None, dx.data_ptr(), *shape, None) == 0
    torch.cuda.synchronize()
    ref_dx = torch.nn.grad.conv3d_input((1, cin) + shape, _w_torch(w, cin, cout), _to_ncdhw(dy, shape), padding=1)
    assert _rel(_to_ncdhw(dx, shape), ref_dx) < 8e-3


def test_unsupported_pair_is_an_error():
    torch = _torch()
    lib = _lib()
    buf = torch.zeros(1024, device="cuda", dtype=torch.bfloat16)
    assert lib.aq_conv3_forward(8, 16, 0, buf.data_ptr(), buf.data_ptr(), None, buf.data_ptr(), 2, 2, 2, None) != 0


def test_umma_and_mma_sync_networks_agree():
    """The network's prediction through the tcgen05 variant against the
    mma.sync variant (the same products; f32 sums in the tensor core's
    order)."""
    torch = _torch()
    lib = _lib()
    import pathlib
    wpath = pathlib.Path(aq.__file__).resolve().parent / "weights" / "unet_64.bin"
    net = aq.UNet(weights=wpath)
    V = 64 ** 3
    g = torch.Generator(device="cuda").manual_seed(9)
    typ = (torch.rand(V, device="cuda", generator=g) < 0.5).to(torch.int8)
    rhs = torch.randn(V, device="cuda", generator=g)
    outs = []
    for impl in (1, 2):
        lib.aq_conv3_set_tiled(impl)
        o = torch.zeros(V, device="cuda")
        net.predict((64, 64, 64), rhs.data_ptr(), typ.data_ptr(), o.data_ptr())
        torch.cuda.synchronize()
        outs.append(o)
    lib.aq_conv3_set_tiled(2)
    _no_umma_timeouts(lib)
    assert _rel(outs[1], outs[0]) < 1e-3
    net.close()
