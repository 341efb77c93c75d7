"""Teacher-forced per-stage comparison of checkers against the reference's
own kernels over many steps, with the tolerance rule for the reference's
racing stages (test infrastructure).

Each stage of each step starts every checker from the reference's state
before that stage (Fluid/Fluid_3D_FLIP.cu:316-352 order), so differences do
not compound.  Rules:

* Stages without a race (G2P + advection, P2G + forces, divergence,
  projection, diffusion): integers bit-exact, floats relative L2 <= 1e-5.
* The sort: the checkers hash with IEEE division, the reference with its
  -use_fast_math division (CMakeLists.txt:16), so a particle within a few
  ulps of a cell face may land in the neighbouring cell.  Every particle
  whose cell differs must be such a particle; particle fields compared by
  pre-sort index are bit-exact (the sort only permutes).
* The in-place Jacobi and extrapolation race (jacobiImpl,
  Fluid/Fluid_3D_kernels.cu:460-505; extrapolateVelocityByOne, :210-422):
  their result depends on which reads see writes of the same launch.  The
  checkers implement the race-free reading (no read sees its own launch's
  writes), one outcome the kernel allows.  The oracle's serial schedule of
  the reference's launch (blocks and warps in launch order, each warp
  reading before writing) is another.  The reference's result must be no
  farther from the checker than those two legal outcomes are from each
  other, with a floor of max(1e-5, 2 x the reference's run-to-run spread)
  for rounding (the reference divides with -use_fast_math).  Components that
  had a velocity before extrapolation must be untouched, bit for bit.
"""
from __future__ import annotations

import numpy as np

from golden_check import STAGE_FIELDS
from scenes import by_original, rel_l2

FLOAT_TOL = 1e-5
RACY = (5, 7)


def _compare(got: dict, ref: dict, fields) -> dict:
    out = {}
    for f in fields:
        if ref[f].dtype.kind in "iu":
            out[f] = int((got[f] != ref[f]).sum())
        else:
            out[f] = rel_l2(got[f], ref[f])
    return out


def hash_face_check(before: dict, got: dict, ref: dict, h: float) -> dict:
    """Particles whose cell differs between checker and reference (by pre-sort
    index), and the largest distance of such a particle to a cell face in
    units of the float spacing of its position / h."""
    si_r, si_g = ref["sort_index"], got["sort_index"]
    hr = np.empty_like(ref["particle_hash"])
    hr[si_r] = ref["particle_hash"]
    hg = np.empty_like(got["particle_hash"])
    hg[si_g] = got["particle_hash"]
    bad = np.nonzero(hr != hg)[0]
    worst = 0.0
    if len(bad):
        q = before["position"][:, bad].astype(np.float32) / np.float32(h)
        dist = np.abs(q.astype(np.float64) - np.round(q.astype(np.float64))) / np.spacing(np.abs(q))
        worst = float(dist.min(axis=0).max())
    perm_equal = all(np.array_equal(by_original(got[f], si_g), by_original(ref[f], si_r))
                     for f in ("position", "velocity_p", "fractions"))
    return {"hash_mismatch": int(len(bad)), "face_ulps": worst, "permuted_fields_equal": perm_equal}


def run(ref, checkers: dict, serial, race_free, steps: int, h: float, log=None) -> list:
    """Teacher-forced records: one dict per (step, stage) with, per checker,
    its comparison to the reference; for the racing stages also the
    reference's spread and the two-schedule envelope."""
    rows = []
    for s in range(steps):
        for k in range(1, 9):
            before = ref.get_state()
            rec = {"s": s, "k": k}
            if k in RACY:  # run-to-run spread of the reference itself
                ref.set_state(before)
                ref.stage(k)
                first = ref.get_state(STAGE_FIELDS[k])
                ref.set_state(before)
            ref.stage(k)
            outs = ref.get_state(STAGE_FIELDS[k])
            got = {}
            for name, chk in checkers.items():
                chk.set_state(before)
                chk.stage(k)
                got[name] = chk.get_state(STAGE_FIELDS[k])
                rec[name] = _compare(got[name], outs, STAGE_FIELDS[k])
                if k == 2:
                    rec[name].update(hash_face_check(before, got[name], outs, h))
                if k == 7:
                    m = before["has_velocity"].astype(bool)
                    sx, sy, sz = ref.size
                    node = ((np.arange(sx)[:, None, None] * (sy + 1) + np.arange(sy)[None, :, None]) * (sz + 1)
                            + np.arange(sz)[None, None, :]).ravel()
                    changed = 0
                    for c in range(3):
                        changed += int((got[name]["new_velocity"][c][node][m[c]] != outs["new_velocity"][c][node][m[c]]).sum())
                    rec[name]["unchanged_mismatch"] = changed
            names = list(checkers)
            for a in range(len(names)):
                for b in range(a + 1, len(names)):
                    rec[f"{names[a]}~{names[b]}"] = _compare(got[names[a]], got[names[b]], STAGE_FIELDS[k])
            if k in RACY:
                rec["spread"] = _compare(first, outs, STAGE_FIELDS[k])
                race_free.set_state(before)
                race_free.stage(k)
                serial.set_state(before)
                serial.stage(k)
                rec["envelope"] = _compare(serial.get_state(STAGE_FIELDS[k]), race_free.get_state(STAGE_FIELDS[k]),
                                           STAGE_FIELDS[k])
            rows.append(rec)
        if log and s % 10 == 0:
            log(s, rows[-4])
    return rows


def judge(rows, checkers, n_particles: int) -> list:
    """Failures of the rules in the module docstring."""
    bad = []
    for r in rows:
        s, k = r["s"], r["k"]
        for name in checkers:
            res = r[name]
            for f, v in res.items():
                if f in ("hash_mismatch", "face_ulps", "permuted_fields_equal", "unchanged_mismatch"):
                    continue
                if k == 2 and f in ("cell_start", "cell_end", "particle_hash", "sort_index", "position",
                                    "velocity_p", "fractions"):
                    continue  # judged through the pre-sort comparison below
                if k in RACY:
                    env, spr = r["envelope"][f], r["spread"][f]
                    if isinstance(v, int):
                        lim = max(2 * spr, env)
                    else:
                        lim = max(FLOAT_TOL, 2 * spr, env)
                    if v > lim:
                        bad.append((s, k, name, f, v, lim))
                elif v > (0 if isinstance(v, int) else FLOAT_TOL):
                    bad.append((s, k, name, f, v))
            if k == 2:
                if not res["permuted_fields_equal"]:
                    bad.append((s, k, name, "permuted_fields"))
                if res["hash_mismatch"] > max(1, n_particles // 10000) or res["face_ulps"] > 4:
                    bad.append((s, k, name, "hash", res["hash_mismatch"], res["face_ulps"]))
                if res["hash_mismatch"] == 0 and any(res[f] for f in ("cell_start", "cell_end", "sort_index")):
                    bad.append((s, k, name, "cell_tables"))
            if k == 7 and res["unchanged_mismatch"]:
                bad.append((s, k, name, "unchanged", res["unchanged_mismatch"]))
        for key, res in r.items():  # checker against checker: ints exact, floats <= 1e-5
            if "~" not in key:
                continue
            for f, v in res.items():
                if v > (0 if isinstance(v, int) else FLOAT_TOL):
                    bad.append((s, k, key, f, v))
    return bad


def summary(rows, checkers) -> dict:
    """Per racing stage and field: the largest checker distance, spread and
    envelope over all steps, and the largest ratio of distance to limit."""
    out = {}
    for k in RACY:
        for r in (x for x in rows if x["k"] == k):
            for f in STAGE_FIELDS[k]:
                key = f"stage{k}/{f}"
                e = out.setdefault(key, {"spread_max": 0, "envelope_min": None, "envelope_max": 0})
                e["spread_max"] = max(e["spread_max"], r["spread"][f])
                env = r["envelope"][f]
                e["envelope_max"] = max(e["envelope_max"], env)
                e["envelope_min"] = env if e["envelope_min"] is None else min(e["envelope_min"], env)
                for name in checkers:
                    v = r[name][f]
                    e[f"{name}_max"] = max(e.get(f"{name}_max", 0), v)
                    lim = max(2 * r["spread"][f], env) if isinstance(v, int) else max(FLOAT_TOL, 2 * r["spread"][f], env)
                    e[f"{name}_worst_fraction_of_limit"] = max(e.get(f"{name}_worst_fraction_of_limit", 0.0),
                                                               (v / lim) if lim > 0 else 0.0)
    for name in checkers:
        h = [r[name]["hash_mismatch"] for r in rows if r["k"] == 2]
        out[f"stage2/{name}_hash_mismatches"] = {"steps_with_any": int(sum(1 for x in h if x)), "total": int(sum(h)),
                                                "max_face_ulps": max(r[name]["face_ulps"] for r in rows if r["k"] == 2)}
    return out
