"""The learned warm start's U-Net, run and trained by the library's kernels,
against the same network written in PyTorch (FP32, the test oracle for the
network): forward pass and the gradients of one training step; and training
on FP64-PCG-labelled systems lowers the held-out pressure error."""
import struct

import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi

pytestmark = pytest.mark.gpu

LAYERS = [(16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (32, 32), (48, 16), (16, 16)]


def _torch():
    import torch
    torch.backends.cudnn.allow_tf32 = False
    torch.backends.cuda.matmul.allow_tf32 = False
    return torch


def read_weights(path):
    raw = open(path, "rb").read()
    magic, version, scale = struct.unpack_from("<IIf", raw, 0)
    assert magic == 0x54454E55 and version == 1
    o = 12
    layers = []
    for cin, cout in LAYERS:
        a, b = struct.unpack_from("<ii", raw, o)
        assert (a, b) == (cin, cout)
        o += 8
        n = 27 * cin * cout
        w = np.frombuffer(raw, np.float32, n, o).reshape(27, cout, cin)
        o += 4 * n
        bias = np.frombuffer(raw, np.float32, cout, o)
        o += 4 * cout
        layers.append((w, bias))
    head = np.frombuffer(raw, np.float32, 17, o)
    return scale, layers, head


class TorchUNet:
    """The network in PyTorch FP32 with the library's bf16-rounded weights."""

    def __init__(self, torch, layers, head, requires_grad=False):
        self.t = torch
        self.params = []
        for w, b in layers:
            cout, cin = w.shape[1], w.shape[2]
            wt = torch.tensor(w, device="cuda").to(torch.bfloat16).float()
            wt = wt.reshape(3, 3, 3, cout, cin).permute(3, 4, 0, 1, 2).contiguous().requires_grad_(requires_grad)
            bt = torch.tensor(b, device="cuda").requires_grad_(requires_grad)
            self.params.append((wt, bt))
        self.hw = torch.tensor(head[:16], device="cuda").requires_grad_(requires_grad)
        self.hb = torch.tensor(head[16:], device="cuda").requires_grad_(requires_grad)

    def __call__(self, x):
        F = self.t.nn.functional

        def c(i, h):
            w, b = self.params[i]
            return F.relu(F.conv3d(h, w, b, padding=1))

        up = lambda h: F.interpolate(h, scale_factor=2, mode="nearest")
        e1 = c(1, c(0, x))
        e2 = c(3, c(2, F.avg_pool3d(e1, 2)))
        b2 = c(5, c(4, F.avg_pool3d(e2, 2)))
        d2 = c(7, c(6, self.t.cat([up(b2), e2], 1)))
        d1 = c(9, c(8, self.t.cat([up(d2), e1], 1)))
        return (d1 * self.hw[None, :, None, None, None]).sum(1)[0] + self.hb[0]

    def grads_in_file_order(self):
        out = []
        for w, b in self.params:
            cout, cin = w.shape[0], w.shape[1]
            out.append(w.grad.permute(2, 3, 4, 0, 1).reshape(27, cout, cin).flatten())
            out.append(b.grad.flatten())
        out += [self.hw.grad, self.hb.grad]
        return [g.detach().cpu().numpy() for g in out]


def apply_A(torch, x, fl):
    """The pressure operator: 6 x_i - sum of the six neighbours, a neighbour
    outside the grid taking x_i (x is 0 off fluid); fluid rows only."""
    xp = torch.nn.functional.pad(x[None, None], (1, 1, 1, 1, 1, 1), mode="replicate")[0, 0]
    s = (xp[2:, 1:-1, 1:-1] + xp[:-2, 1:-1, 1:-1] + xp[1:-1, 2:, 1:-1] + xp[1:-1, :-2, 1:-1]
         + xp[1:-1, 1:-1, 2:] + xp[1:-1, 1:-1, :-2])
    return torch.where(fl, 6 * x - s, torch.zeros_like(x))


def apply_J(torch, x, fl, k):
    """k homogeneous Jacobi sweeps: the mean of the six neighbours (clamped at
    the walls) on fluid cells, 0 elsewhere."""
    for _ in range(k):
        xp = torch.nn.functional.pad(x[None, None], (1, 1, 1, 1, 1, 1), mode="replicate")[0, 0]
        s = (xp[2:, 1:-1, 1:-1] + xp[:-2, 1:-1, 1:-1] + xp[1:-1, 2:, 1:-1] + xp[1:-1, :-2, 1:-1]
             + xp[1:-1, 1:-1, 2:] + xp[1:-1, 1:-1, :-2])
        x = torch.where(fl, s / 6, torch.zeros_like(x))
    return x


def _input(torch, rhs, typ, shape):
    x = torch.zeros(1, 16, *shape, device="cuda")
    x[0, 0] = torch.tensor(rhs.reshape(shape), device="cuda").to(torch.bfloat16).float()
    x[0, 1] = torch.tensor((typ.reshape(shape) == 1).astype(np.float32), device="cuda")
    return x


def _dataset(shape, n_scenes=3, steps=(2, 5, 9), seed=3):
    ds = aq.Dataset(shape, capacity=n_scenes * len(steps))
    rng = np.random.RandomState(seed)
    for k in range(n_scenes):
        vols = [dict(shape="box", min=(0, 0, 0), max=(1, float(rng.uniform(0.15, 0.4)), 1)),
                dict(shape="sphere", center=tuple(float(v) for v in rng.uniform(0.3, 0.7, 3)),
                     radius=float(rng.uniform(0.1, 0.2)))]
        cfg = _abi.make_config(shape, vols, timestep=0.01, pressure_iterations=60, seed=k + 1)
        with aq.Fluid(cfg) as f:
            done = 0
            for s in steps:
                f.step(s - done)
                done = s
                for stage in range(1, 5):  # rebuild the system of the next step
                    f.run_stage(stage)
                ds.add_fluid(f, 1e-10)
                for stage in range(5, 9):
                    f.run_stage(stage)
                done += 1
    return ds


def test_forward_matches_torch(tmp_path):
    torch = _torch()
    shape = (16, 12, 20)
    net = aq.UNet(seed=5)
    net.save(tmp_path / "w.bin")
    scale, layers, head = read_weights(tmp_path / "w.bin")
    V = int(np.prod(shape))
    rng = np.random.RandomState(1)
    typ = (rng.rand(V) < 0.6).astype(np.int8)
    rhs = (rng.randn(V) * (typ == 1)).astype(np.float32)
    t_rhs = torch.tensor(rhs, device="cuda")
    t_typ = torch.tensor(typ, device="cuda")
    out = torch.zeros(V, device="cuda")
    torch.cuda.synchronize()
    net.predict(shape, t_rhs.data_ptr(), t_typ.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    m = float(np.abs(rhs).max())
    ref = TorchUNet(torch, layers, head)(_input(torch, rhs / m, typ, shape)).flatten() * m * scale
    fl = t_typ == 1
    got, want = out[fl], ref[fl]
    assert float((got - want).norm() / want.norm()) < 3e-2  # bf16 activations vs f32
    assert float(out[~fl].abs().max()) == 0.0


def test_training_gradients_match_torch(tmp_path):
    torch = _torch()
    shape = (16, 16, 16)
    ds = _dataset(shape, n_scenes=1, steps=(3,))
    net = aq.UNet(seed=9)
    net.save(tmp_path / "w.bin")
    _, layers, head = read_weights(tmp_path / "w.bin")
    alpha, k = 0.5, 3
    net.train(ds, 0, 1, steps=1, lr=0.0, out_scale=1.0, residual_weight=alpha, residual_sweeps=k)
    got = net.gradients()
    s = ds.get(0)
    ref = TorchUNet(torch, layers, head, requires_grad=True)
    out = ref(_input(torch, s["rhs"], s["type"], shape))
    fl = torch.tensor(s["type"] == 1, device="cuda").reshape(shape)
    tgt = torch.tensor(s["target"], device="cuda").reshape(shape)
    e = torch.where(fl, out - tgt, torch.zeros_like(out))
    tz = torch.where(fl, tgt, torch.zeros_like(tgt))
    AJ = lambda x: apply_A(torch, apply_J(torch, x, fl, k), fl)
    loss = (e ** 2).sum() / (tgt[fl] ** 2).sum() + alpha * (AJ(e) ** 2).sum() / (AJ(tz) ** 2).sum()
    loss.backward()
    o = 0
    for i, g_ref in enumerate(ref.grads_in_file_order()):
        g = got[o:o + g_ref.size]
        o += g_ref.size
        cos = float(np.dot(g, g_ref) / (np.linalg.norm(g) * np.linalg.norm(g_ref) + 1e-30))
        ratio = float(np.linalg.norm(g) / (np.linalg.norm(g_ref) + 1e-30))
        assert cos > 0.98 and 0.9 < ratio < 1.1, (i, cos, ratio)
    assert o == got.size


def test_training_lowers_held_out_error(tmp_path):
    shape = (16, 16, 16)
    ds = _dataset(shape, n_scenes=4, steps=(2, 6, 10))
    n = len(ds)
    assert n == 12
    net = aq.UNet(seed=2)
    net.train(ds, 0, 9, steps=1, lr=0.0)  # sets the output scale only
    before = net.evaluate(ds, 9, 3)
    net.train(ds, 0, 9, steps=400, lr=2e-3, seed=4)
    after = net.evaluate(ds, 9, 3)
    assert after < 0.7 * before, (before, after)
    assert after < 0.8, (before, after)
    net.save(tmp_path / "t.bin")
    other = aq.UNet(seed=99, weights=tmp_path / "t.bin")
    assert other.evaluate(ds, 9, 3) == pytest.approx(after, rel=1e-6)
