"""Particle-only solvers (PBF, PCISPH) through the C ABI.

The library's kernels round every operation as the reference writes it and
walk neighbours in the reference's order, as the CPU oracle does: seeding,
rest densities and whole steps equal the oracle's bit for bit.  Against the
reference's own solvers (recorded fixtures, and live where
oracle/_ref/libaqsph.so is present) steps are teacher-forced and judged by
golden_check.judge_sph_step.
"""
import numpy as np
import pytest

import aquarius_b200 as aq
from aquarius_b200 import _abi
from golden_check import judge_sph_step, load_sph, sph_config_from_bytes, sph_fixture_state
from oracle_binding import RefSph, SphOracle, sph_ref_available

pytestmark = pytest.mark.gpu

METHODS = {"pbf": _abi.SPH_PBF, "pcisph": _abi.SPH_PCISPH}
FIELDS = {
    "pbf": ["position", "velocity", "density", "rest_density", "last_position", "lambda"],
    "pcisph": ["position", "velocity", "density", "rest_density", "pressure", "pressure_force",
               "predicted_position", "predicted_velocity"],
}


@pytest.mark.parametrize("method", ["pbf", "pcisph"])
@pytest.mark.parametrize("budget", [8000, 30000, 300000])
def test_init_and_steps_match_oracle_bitwise(method, budget):
    cfg = _abi.sph_config(METHODS[method], max_particle_count=budget)
    s, o = aq.Sph(cfg), SphOracle(cfg)
    assert s.n == o.n > 0
    assert (s.spacing, s.kernel_radius, s.grid) == (o.spacing, o.kernel_radius, o.grid)
    steps = 3 if budget < 300000 else 1
    for k in range(steps + 1):
        if k:
            s.step(1)
            o.step(1)
        a, b = s.get_state(FIELDS[method]), o.get_state(FIELDS[method])
        for f in FIELDS[method]:
            np.testing.assert_array_equal(a[f], b[f], err_msg=f"{method} step {k} {f}")


@pytest.mark.parametrize("method", ["pbf", "pcisph"])
def test_steps_in_one_call_equal_steps_one_by_one(method):
    cfg = _abi.sph_config(METHODS[method], max_particle_count=30000)
    a, b = aq.Sph(cfg), aq.Sph(cfg)
    a.step(3)
    for _ in range(3):
        b.step(1)
    sa, sb = a.get_state(FIELDS[method]), b.get_state(FIELDS[method])
    for f in FIELDS[method]:
        np.testing.assert_array_equal(sa[f], sb[f], err_msg=f)
    assert abs(sa["physical_time"] - 3 * cfg.timestep) < 1e-9


@pytest.mark.parametrize("method", ["pbf", "pcisph"])
def test_uploaded_state_steps_like_the_oracle(method):
    """State injection: an oracle state after two steps, uploaded unsorted
    (every step starts with the spatial hash), then one step on each."""
    cfg = _abi.sph_config(METHODS[method], max_particle_count=30000)
    o = SphOracle(cfg)
    o.step(2)
    st = o.get_state()
    perm = np.random.default_rng(5).permutation(o.n)
    shuffled = {k: (v[..., perm] if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    s = aq.Sph(cfg)
    s.set_state(shuffled)
    o2 = SphOracle(cfg)
    o2.set_state(shuffled)
    s.step(1)
    o2.step(1)
    a, b = s.get_state(FIELDS[method]), o2.get_state(FIELDS[method])
    for f in FIELDS[method]:
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


def test_positions_outside_the_container_are_rejected():
    s = aq.Sph(_abi.sph_config(_abi.SPH_PBF, max_particle_count=8000))
    st = s.get_state(["position"])
    st["position"][1, 0] = -1.0
    with pytest.raises(aq.AquariusError):
        s.set_state(st)


@pytest.mark.parametrize("method", ["pbf", "pcisph"])
def test_against_reference_fixtures(method):
    data = load_sph()
    if data is None:
        pytest.skip("fixture missing")
    cfg = sph_config_from_bytes(data[f"{method}/config"])
    s = aq.Sph(cfg)
    s0 = sph_fixture_state(data, method, 0)
    st = s.get_state()
    np.testing.assert_array_equal(st["position"], s0["position"])
    for k in range(3):
        s.set_state(sph_fixture_state(data, method, k))
        s.step(1)
        assert judge_sph_step(method, s.get_state(), sph_fixture_state(data, method, k + 1)) == [], k


@pytest.mark.skipif(not sph_ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("method", ["pbf", "pcisph"])
def test_against_live_reference(method):
    cfg = _abi.sph_config(METHODS[method], max_particle_count=30000)
    r = RefSph(cfg)
    s = aq.Sph(cfg)
    assert (r.n, r.grid) == (s.n, s.grid)
    np.testing.assert_array_equal(s.get_state(["position"])["position"], r.get_state(["position"])["position"])
    for k in range(3):
        r.step(1)
        st = r.get_state()
        s.set_state(st)
        r.step(1)
        s.step(1)
        assert judge_sph_step(method, s.get_state(), r.get_state()) == [], k
    r.close()


@pytest.mark.skipif(not sph_ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("method", ["pbf", "pcisph"])
def test_step_time_vs_reference(method, capsys):
    """Budget 3e6 (about 590k particles) on the same GPU: the best host wall
    time of five single steps, ours (one graph launch, then a synchronize)
    against the reference's (its kernels and its own synchronisations)."""
    import time

    cfg = _abi.sph_config(METHODS[method], max_particle_count=3000000)
    s = aq.Sph(cfg)
    s.step(2)
    s.synchronize()
    reps = 5

    def best(step):
        times = []
        for _ in range(reps):
            t0 = time.perf_counter()
            step()
            times.append(time.perf_counter() - t0)
        return min(times)

    ours = best(lambda: (s.step(1), s.synchronize()))
    r = RefSph(cfg)
    r.step(2)
    ref = best(lambda: r.step(1))  # the harness synchronises after the step
    r.close()
    with capsys.disabled():
        print(f"\n{method} budget 3e6 ({s.n} particles): ours {ours * 1e3:.2f} ms/step, "
              f"reference {ref * 1e3:.2f} ms/step")
    assert ours < ref
