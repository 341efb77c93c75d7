"""BASELINE config 1 parity: the 50^3 ball drop (pool y < 0.2, sphere r 0.15
at (0.5, 0.65, 0.5), 8 particles per cell, dt 0.01, FLIP 0.95, 100 Jacobi
sweeps, pressure carried as the reference does) for 100 steps, every stage
teacher-forced from the reference's own kernels (oracle/_ref/libaqref.so,
Fluid/Fluid_3D_FLIP.cu:316-352) and compared for the CUDA library and the
CPU oracle under the rules of racy_envelope.py.  50 is not a multiple of 4,
so the library runs its tiled sweep kernels here.

Also the headline size: one teacher-forced step of BASELINE config 2 (128^3,
Jacobi to relative residual 1e-4 capped at 2000, zero-init pressure), the
library against the oracle on every field of every stage."""
import json
import os
import pathlib

import numpy as np
import pytest

import oracle_binding
import racy_envelope
from aquarius_b200 import _abi
from golden_check import STAGE_FIELDS
from lib_checker import LibChecker
from oracle_binding import Oracle, RefFluid
from scenes import ball_drop, rel_l2

pytestmark = pytest.mark.gpu

CFG1_STEPS = 100


def config1():
    return ball_drop((50, 50, 50), pool=0.2, center=(0.5, 0.65, 0.5), radius=0.15, dt=0.01, flip_coeff=0.95,
                     pressure_iterations=100, pressure_init=_abi.PRESSURE_CARRY)


@pytest.mark.skipif(not oracle_binding.ref_available(), reason="oracle/_ref not built")
def test_config1_100_steps_teacher_forced_against_reference():
    cfg = config1()
    ref = RefFluid(cfg)
    checkers = {"library": LibChecker(cfg), "oracle": Oracle(cfg)}
    serial = Oracle(cfg)
    serial.set_schedule(True)
    race_free = checkers["oracle"]
    h = cfg.domain_size / cfg.size_y
    rows = racy_envelope.run(ref, checkers, serial, race_free, CFG1_STEPS, h)
    summ = racy_envelope.summary(rows, checkers)
    print(json.dumps(summ, indent=1))
    out = os.environ.get("AQ_CFG1_SUMMARY")
    if out:
        pathlib.Path(out).write_text(json.dumps(summ, indent=1) + "\n")
    bad = racy_envelope.judge(rows, checkers, ref.n)
    assert bad == [], bad[:20]
    # the library's stages equal the oracle's bit for bit where both are exact
    for r in rows:
        for f, v in r["library~oracle"].items():
            if r["k"] in (2, 4, 5, 7, 8) or isinstance(v, int):
                assert v == 0, (r["s"], r["k"], f, v)
    ref.close()
    checkers["library"].f.close()
    for o in (checkers["oracle"], serial):
        o.close()


def test_config2_128_teacher_forced_step_against_oracle():
    vols = [dict(shape="box", min=(0, 0, 0), max=(1, 0.3, 1), phase=0),
            dict(shape="sphere", center=(0.5, 0.7, 0.5), radius=0.12, phase=0)]
    cfg = _abi.make_config((128, 128, 128), vols, timestep=0.005, flip_coeff=0.95, particle_jitter=0.05,
                           pressure_init=_abi.PRESSURE_ZERO, solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=1e-4,
                           max_iterations=2000, check_interval=40)
    orc = Oracle(cfg)
    lib = LibChecker(cfg)
    orc.step(2)  # a moving state: the third step is compared stage by stage
    for k in range(1, 9):
        before = orc.get_state()
        orc.stage(k)
        want = orc.get_state(STAGE_FIELDS[k])
        lib.set_state(before)
        lib.stage(k)
        got = lib.get_state(STAGE_FIELDS[k])
        for f in STAGE_FIELDS[k]:
            if want[f].dtype.kind in "iu":
                assert np.array_equal(got[f], want[f]), (k, f, int((got[f] != want[f]).sum()))
            else:
                e = rel_l2(got[f], want[f])
                assert e <= 1e-5, (k, f, e)
                if k in (2, 4, 5, 7, 8):  # same arithmetic in the same order
                    assert np.array_equal(got[f], want[f]), (k, f, e)
        if k == 5:
            assert lib.f.solve_stats()["iterations"] == orc.solve_stats()["iterations"]
    lib.f.close()
    orc.close()
