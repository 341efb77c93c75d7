"""AQ_PRESSURE_LEARNED: the network's prediction warm-starts the Jacobi solve,
20 sweeps from it are compared with 20 sweeps from zero (the fallback and the
judge), and the solve continues from the better start.  Checked against
plain zero-init fluids on the same system, graph against eager, and with a
network trained for the test scene against an untrained one."""
import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi
from test_unet_gpu import _dataset

pytestmark = pytest.mark.gpu

SHAPE = (32, 32, 32)


def _cfg(init, mode=_abi.SOLVE_RESIDUAL, **kw):
    vols = [dict(shape="box", min=(0, 0, 0), max=(1, 0.3, 1)),
            dict(shape="sphere", center=(0.5, 0.7, 0.5), radius=0.15)]
    base = dict(timestep=0.01, pressure_init=init, solve_mode=mode, rel_residual=1e-4, max_iterations=400,
                check_interval=40, pressure_iterations=20)
    base.update(kw)
    return _abi.make_config(SHAPE, vols, **base)


@pytest.fixture(scope="module")
def trained_net():
    # systems of this scene's first steps (and of a few other seeded scenes)
    ds = aq.Dataset(SHAPE, capacity=24)
    with aq.Fluid(_cfg(_abi.PRESSURE_ZERO, _abi.SOLVE_FIXED, pressure_iterations=200)) as f:
        for _ in range(12):
            for stage in range(1, 5):
                f.run_stage(stage)
            ds.add_fluid(f, 1e-10)
            for stage in range(5, 9):
                f.run_stage(stage)
    other = _dataset(SHAPE, n_scenes=2, steps=(2, 6, 10))
    net = aq.UNet(seed=3)
    net.train(ds, 0, len(ds), steps=600, lr=2e-3, seed=5)
    del other
    return net


def test_learned_needs_a_network():
    with aq.Fluid(_cfg(_abi.PRESSURE_LEARNED)) as f:
        with pytest.raises(aq.AquariusError, match="needs a network"):
            f.step(1)


def test_zero_path_is_the_plain_zero_init_solve(trained_net):
    # first step: identical systems; the fallback path is a plain 20-sweep zero-init solve
    with aq.Fluid(_cfg(_abi.PRESSURE_LEARNED)) as f, \
            aq.Fluid(_cfg(_abi.PRESSURE_ZERO, _abi.SOLVE_FIXED, pressure_iterations=20)) as z:
        f.set_warm_start(trained_net)
        f.step(1)
        z.step(1)
        s, sz = f.solve_stats(), z.solve_stats()
        assert s["zero_rel_residual"] == sz["rel_residual"]
        assert s["warm_start"] in (1, 2)
        if s["warm_start"] == 1:
            assert s["warm_rel_residual"] <= s["zero_rel_residual"]
        else:
            assert s["warm_rel_residual"] > s["zero_rel_residual"]
        assert s["iterations"] >= 20 + 40 and s["iterations"] % 40 == 20


def test_trained_network_beats_zero_start(trained_net):
    with aq.Fluid(_cfg(_abi.PRESSURE_LEARNED)) as f:
        f.set_warm_start(trained_net)
        kept = 0
        for _ in range(6):
            f.step(1)
            s = f.solve_stats()
            kept += s["warm_start"] == 1
        assert kept >= 4, s  # the trained prediction wins most steps
        assert s["warm_rel_residual"] < s["zero_rel_residual"]


def test_untrained_network_falls_back():
    net = aq.UNet(seed=11)
    with aq.Fluid(_cfg(_abi.PRESSURE_LEARNED)) as f:
        f.set_warm_start(net)
        f.step(2)
        s = f.solve_stats()
        assert s["warm_start"] == 2 and s["warm_rel_residual"] > s["zero_rel_residual"]


def test_learned_graph_equals_eager(trained_net):
    out = []
    for graph in (True, False):
        with aq.Fluid(_cfg(_abi.PRESSURE_LEARNED)) as f:
            f.set_warm_start(trained_net)
            f.set_graph_mode(graph)
            f.step(3)
            st = f.download_state(["pressure", "position"])
            out.append((st, f.solve_stats()))
    (a, sa), (b, sb) = out
    np.testing.assert_array_equal(a["pressure"], b["pressure"])
    np.testing.assert_array_equal(a["position"], b["position"])
    assert sa["iterations"] == sb["iterations"] and sa["warm_start"] == sb["warm_start"]


def test_evaluate_warm_matches_the_step_pick(trained_net):
    # the dataset-side ratio (J^20 applied to the prediction's error against
    # the FP64 solution) equals the step's residual ratio after 20 sweeps
    ds = aq.Dataset(SHAPE, capacity=1)
    with aq.Fluid(_cfg(_abi.PRESSURE_ZERO, _abi.SOLVE_FIXED, pressure_iterations=200)) as z:
        for stage in range(1, 5):
            z.run_stage(stage)
        ds.add_fluid(z, 1e-12)
    ratio = trained_net.evaluate_warm(ds, 0, 1, 20)
    with aq.Fluid(_cfg(_abi.PRESSURE_LEARNED)) as f:
        f.set_warm_start(trained_net)
        f.step(1)
        s = f.solve_stats()
    assert ratio == pytest.approx(s["warm_rel_residual"] / s["zero_rel_residual"], rel=2e-2)
