"""Multiphase runs: the per-phase concentration mass (sum of the particles'
volume fractions, FP64) against the CPU oracle's, and the single-phase case
(the particle count).  The change of this sum over a run is the
concentration-mass conservation error of multiphase diffusion."""
import numpy as np
import pytest

import aquarius_b200 as aq
from oracle_binding import Oracle
from scenes import SCENES

pytestmark = pytest.mark.gpu


def test_phase_mass_matches_oracle_fractions():
    cfg = SCENES["multi_16"]()
    f, o = aq.Fluid(cfg), Oracle(cfg)
    for _ in range(3):
        f.step(1)
        o.step(1)
        m = np.array(f.phase_mass())
        fr = o.get_state(["fractions"])["fractions"].reshape(4, -1).astype(np.float64)
        np.testing.assert_allclose(m, fr.sum(axis=1), rtol=1e-5, atol=1e-3)
    assert abs(sum(m) - f.particleCount) <= 1e-3 * f.particleCount  # fractions are normalised
    f.close()


def test_single_phase_mass_is_the_particle_count():
    cfg = SCENES["cfg1_16"]()
    with aq.Fluid(cfg) as f:
        f.step(2)
        m = f.phase_mass()
        assert m[cfg.volumes[0].phase] == f.particleCount and sum(m) == f.particleCount
