"""Generates the golden fixtures in tests/golden/ from the reference's own
FLIP kernels (oracle/_ref/libaqref.so, built headless by `make -C oracle ref`
where the reference sources are present).  Needs a GPU.

    python tests/golden/make_golden.py --out tests/golden

For each scene it records the reference's init state and, for every stage of
the first steps, the fields that stage writes, starting each stage from the
reference's own state (teacher forcing).  It also records:
  * the texture address probe: what the reference's tex3D returns for
    out-of-range y/z coordinates (createField3D sets only addressMode[0],
    Fluid/VolumeData.cuh:58-67);
  * the reference's run-to-run spread per stage (its Jacobi, diffusion and
    extrapolation kernels update in place and race);
  * ink particles (ref_ink.npz), through the reference's own initInkRenderer /
    transferToInkParticles / moveInkParticles, which its Fluid leaves
    switched off: the seeded count and a SHA-256 of all seeded positions,
    and, for a fixed sample of ink particles, the ink before and after the
    advance that would end each step, with the grids it read.

    python tests/golden/make_golden.py --out tests/golden --only ink
  * the surface mesher (ref_mesh.npz, texture_linear_probe.npz), through the
    reference's own Mesher (oracle/_ref/libaqmesh.so) on the particles of the
    recorded FLIP fixtures after their last sort: the SDF grid, the occupied
    cube count and aggregates of all cube records, and a sample of records;
    and what the SDF's texture settings (linear filter, border in x) return
    at chosen coordinates of a random field.

    python tests/golden/make_golden.py --out tests/golden --only mesh
  * the particle-only solvers (ref_sph.npz), through the reference's own
    Fluid_3D_PBF / Fluid_3D_PCISPH (oracle/_ref/libaqsph.so) on small
    seeded configs: the state after init and after each of three steps.

    python tests/golden/make_golden.py --out tests/golden --only sph
  * the shading of the headless frame (ref_shade.npz), through the
    reference's own fragment shaders and camera compiled as C++ on the CPU
    (oracle/_ref/libaqshade.so, `make -C oracle shade`; no GPU): the default
    camera's matrices for several windows, and seeded fragments of
    FluidMeshRenderer_fs (every mesh mode and environment),
    RayTraceEnvironment and Container_face_fs with their outputs.

    python tests/golden/make_golden.py --out tests/golden --only shade
"""
from __future__ import annotations

import argparse
import ctypes as ct
import hashlib
import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from aquarius_b200 import _abi  # noqa: E402
from oracle_binding import RefFluid, RefMesher, RefSph, probe_linear, probe_texture  # noqa: E402
from scenes import SCENES, rel_l2  # noqa: E402
from mesh_check import canonical_records, record_aggregates  # noqa: E402

STAGE_FIELDS = {
    1: ["position", "velocity_p", "fractions"],
    2: ["position", "velocity_p", "fractions", "cell_start", "cell_end", "particle_hash", "sort_index"],
    3: ["content", "velocity", "new_velocity", "density", "volume_fractions", "new_volume_fractions"],
    4: ["particle_count_cell", "divergence"],
    5: ["pressure"],
    6: ["new_velocity", "has_velocity"],
    7: ["new_velocity", "has_velocity"],
    8: ["new_volume_fractions"],
}

GOLDEN_SCENES = {"cfg1_16": 2, "aniso": 1, "multi_16": 1}
INK_SCENES = {"cfg1_16": 2, "aniso": 2}
INK_SAMPLE = 2048


def record_scene(name: str, steps: int) -> dict:
    cfg = SCENES[name]()
    ref = RefFluid(cfg)
    out = {"config": np.frombuffer(bytes(cfg), dtype=np.uint8).copy()}
    st = ref.get_state()
    for k, v in st.items():
        if k != "physical_time":
            out[f"init/{k}"] = v
    spread = {}
    for s in range(steps):
        for k in range(1, 9):
            before = ref.get_state()
            ref.stage(k)
            after = ref.get_state()
            for f in STAGE_FIELDS[k]:
                out[f"s{s}/k{k}/{f}"] = after[f]
            # run-to-run spread: replay the stage from the same state, then
            # continue from the first run (the one recorded above)
            ref.set_state(before)
            ref.stage(k)
            again = ref.get_state(STAGE_FIELDS[k])
            for f in STAGE_FIELDS[k]:
                if after[f].dtype.kind == "f":
                    spread[f"s{s}/k{k}/{f}"] = rel_l2(again[f], after[f])
                else:
                    spread[f"s{s}/k{k}/{f}"] = int((again[f] != after[f]).sum())
            ref.set_state(after)
    ref.close()
    return out, spread


def record_special() -> dict:
    """Race-free settings of the reference's in-place kernels.

    jacobi_converged: 3000 in-place sweeps from the state after stage 4; the
        racy sweep order no longer matters at the fixed point, which pins the
        operator (coefficients, rhs, walls, air).
    jacobi_isolated: one sweep where every fluid cell is surrounded by air
        with p = 0, so no cell reads a value written in the same sweep.
    extrap_isolated: extrapolation where every cell lacking a component is
        surrounded by cells that have it; those never change, so the pass
        reads no value written in the same pass.
    """
    out = {}
    rng = np.random.default_rng(7)
    cfg = SCENES["cfg1_16"](pressure_iterations=3000)
    ref = RefFluid(cfg)
    for k in range(1, 5):
        ref.stage(k)
    st = ref.get_state()
    out["jacobi_converged/config"] = np.frombuffer(bytes(cfg), dtype=np.uint8).copy()
    for f, v in st.items():
        if f != "physical_time":
            out[f"jacobi_converged/in/{f}"] = v
    ref.stage(5)
    out["jacobi_converged/out/pressure"] = ref.get_state(["pressure"])["pressure"]
    ref.close()

    cfg = SCENES["cfg1_16"](pressure_iterations=1)
    ref = RefFluid(cfg)
    st = ref.get_state()
    sx, sy, sz = cfg.size_x, cfg.size_y, cfg.size_z
    x, y, z = np.meshgrid(np.arange(sx + 1), np.arange(sy + 1), np.arange(sz + 1), indexing="ij")
    inner = (x < sx) & (y < sy) & (z < sz)
    iso = ((x + 2 * y + 4 * z) % 8 == 3) & inner
    content = st["content"].reshape(sx + 1, sy + 1, sz + 1).copy()
    content[inner] = 0
    content[iso] = 1
    st["content"] = content.ravel().astype(np.int32)
    st["pressure"] = np.zeros_like(st["pressure"])
    st["divergence"] = rng.uniform(-1, 1, st["divergence"].shape).astype(np.float32)
    st["density"] = rng.uniform(0.5, 2, st["density"].shape).astype(np.float32)
    ref.set_state(st)
    ref.stage(5)
    out["jacobi_isolated/config"] = np.frombuffer(bytes(cfg), dtype=np.uint8).copy()
    for f in ["content", "pressure", "divergence", "density"]:
        out[f"jacobi_isolated/in/{f}"] = st[f]
    out["jacobi_isolated/out/pressure"] = ref.get_state(["pressure"])["pressure"]

    st = ref.get_state()
    nv = rng.uniform(-2, 2, st["new_velocity"].shape).astype(np.float32)
    has = np.ones_like(st["has_velocity"])
    xc, yc, zc = np.meshgrid(np.arange(sx), np.arange(sy), np.arange(sz), indexing="ij")
    # With S = x + 2y + 4z, component a lacks velocity where S = r[a] (mod 8).
    # A neighbour along axis d sits at S +- (1, 2, 4)[d]; the residues below
    # keep every neighbour a hole reads (its averaged component and its
    # velocity along the neighbour direction) out of the holes, so no value
    # read in a pass is written in that pass.
    residue = (0, 3, 2)
    for comp in range(3):
        holes = ((xc + 2 * yc + 4 * zc) % 8 == residue[comp]).ravel()
        has[comp][holes] = 0
    st["new_velocity"] = nv
    st["has_velocity"] = has.astype(np.int32)
    ref.set_state(st)
    ref.stage(7)
    got = ref.get_state(["new_velocity", "has_velocity"])
    out["extrap_isolated/config"] = np.frombuffer(bytes(cfg), dtype=np.uint8).copy()
    for f in ["new_velocity", "has_velocity", "content"]:
        out[f"extrap_isolated/in/{f}"] = st[f]
    out["extrap_isolated/out/new_velocity"] = got["new_velocity"]
    out["extrap_isolated/out/has_velocity"] = got["has_velocity"]
    ref.close()
    return out


def record_ink() -> dict:
    out = {}
    for name, steps in INK_SCENES.items():
        cfg = SCENES[name]()
        ref = RefFluid(cfg)
        n = ref.enable_ink()  # right after init: continues the seeding's rand() sequence
        pos = ref.get_ink()["position"]
        idx = np.unique(np.linspace(0, n - 1, INK_SAMPLE).astype(np.int64))
        out[f"{name}/config"] = np.frombuffer(bytes(cfg), dtype=np.uint8).copy()
        out[f"{name}/count"] = np.int64(n)
        out[f"{name}/init_sha256"] = np.frombuffer(hashlib.sha256(pos.tobytes()).digest(), np.uint8).copy()
        out[f"{name}/sample"] = idx
        out[f"{name}/init_position"] = pos[:, idx]
        for s in range(steps):
            ref.step(1)
            st = ref.get_state(["velocity", "new_velocity"])
            before = ref.get_ink()
            ref.ink_advance()
            after = ref.get_ink()
            out[f"{name}/s{s}/velocity"] = st["velocity"]
            out[f"{name}/s{s}/new_velocity"] = st["new_velocity"]
            for k in ("position", "velocity"):
                out[f"{name}/s{s}/in_{k}"] = before[k][:, idx]
                out[f"{name}/s{s}/out_{k}"] = after[k][:, idx]
        ref.close()
    return out


MESH_SCENES = {"cfg1_16": "s1/k2/position", "aniso": "s0/k2/position"}
MESH_SAMPLE = 1024


def record_mesh() -> dict:
    out = {}
    for name, key in MESH_SCENES.items():
        fx = np.load(HERE / f"ref_{name}.npz")
        cfg = SCENES[name]()
        pos = fx[key]
        h = float(np.float32(cfg.domain_size) / np.float32(cfg.size_y))  # Fluid_3D_FLIP.cu:444
        m = RefMesher((cfg.size_x, cfg.size_y, cfg.size_z), h, pos.shape[1])
        r = m.mesh(pos)
        recs = canonical_records(r["records"])
        idx = np.unique(np.linspace(0, len(recs) - 1, MESH_SAMPLE).astype(np.int64))
        out[f"{name}/input"] = np.array(key)
        out[f"{name}/sdf_size"] = np.array(m.sdf_size)
        out[f"{name}/mesh_size"] = np.array(m.mesh_size)
        out[f"{name}/cell"] = np.array([m.h_sdf, m.h_mesh], np.float32)
        out[f"{name}/sdf"] = r["sdf"]
        out[f"{name}/cubes"] = np.int64(r["cubes"])
        for k, v in record_aggregates(r["records"]).items():
            out[f"{name}/agg/{k}"] = np.asarray(v)
        out[f"{name}/sample"] = recs[idx]
        m.close()
        print(name, "mesh:", r["cubes"], "cubes, sdf", m.sdf_size)
    return out


SPH_STEPS = 3


def sph_scenes() -> dict:
    """Small seeded configs of the two solvers (about 1,700 particles)."""
    return {"pbf": _abi.sph_config(_abi.SPH_PBF, max_particle_count=8000),
            "pcisph": _abi.sph_config(_abi.SPH_PCISPH, max_particle_count=8000)}


def record_sph() -> dict:
    out = {}
    for name, cfg in sph_scenes().items():
        ref = RefSph(cfg)
        out[f"{name}/config"] = np.frombuffer(bytes(cfg), dtype=np.uint8).copy()
        out[f"{name}/info"] = np.array([ref.spacing, ref.kernel_radius], np.float32)
        out[f"{name}/grid"] = np.array(ref.grid)
        for s in range(SPH_STEPS + 1):
            if s:
                ref.step(1)
            st = ref.get_state()
            for k, v in st.items():
                if k != "physical_time":
                    out[f"{name}/s{s}/{k}"] = v
        print(name, "sph:", ref.n, "particles")
        ref.close()
    return out


def record_linear_probe() -> dict:
    rng = np.random.default_rng(11)
    w, h, d = 7, 6, 5
    vals = rng.uniform(-1, 1, (d, h, w)).astype(np.float32)
    rnd = np.stack([rng.uniform(-1.5, w + 1.5, 3000), rng.uniform(-1.5, h + 1.5, 3000),
                    rng.uniform(-1.5, d + 1.5, 3000)], 1)
    t = 1.0 + np.arange(2048) / 2048.0  # x fractions at 1/2048 steps: pins the weight quantisation
    sweep = np.stack([t, np.full_like(t, 2.5), np.full_like(t, 2.5)], 1)
    coords = np.concatenate([rnd, sweep]).astype(np.float32)
    return {"values": vals, "coords": coords, "out": probe_linear(vals, coords)}


def texture_probe() -> dict:
    w, h, d = 6, 5, 4
    coords = [(2, -1, 2), (2, h, 2), (2, 2, -1), (2, 2, d), (-1, 2, 2), (w, 2, 2), (2, h - 1, 2), (2, 0, 2),
              (2, 2, d - 1), (2, 2, 0), (0, 2, 2), (w - 1, 2, 2)]
    vals = probe_texture(w, h, d, coords)
    field = lambda x, y, z: float(x + 100 * y + 10000 * z)
    res = {"extent": [w, h, d], "reads": [[list(c), float(v)] for c, v in zip(coords, vals)]}

    def mode(v, clamp, wrap):
        if v == clamp:
            return "clamp"
        if v == wrap:
            return "wrap"
        if v == 0.0:
            return "border"
        return f"other({v})"
    res["y_low"] = mode(vals[0], field(2, 0, 2), field(2, h - 1, 2))
    res["y_high"] = mode(vals[1], field(2, h - 1, 2), field(2, 0, 2))
    res["z_low"] = mode(vals[2], field(2, 2, 0), field(2, 2, d - 1))
    res["z_high"] = mode(vals[3], field(2, 2, d - 1), field(2, 2, 0))
    res["x_low"] = mode(vals[4], field(0, 2, 2), field(w - 1, 2, 2))
    res["x_high"] = mode(vals[5], field(w - 1, 2, 2), field(0, 2, 2))
    return res


SHADE_WINDOWS = [(1728, 864, 10.0), (320, 160, 10.0), (97, 31, 3.5), (1000, 1000, 7.25)]


def record_shade() -> dict:
    from oracle_binding import RenderOracle
    lib = ct.CDLL(str(ROOT / "oracle" / "_ref" / "libaqshade.so"))
    P, I = ct.c_void_p, ct.c_int32
    lib.aqshade_camera.argtypes = [I, I, ct.c_float, P, P, P]
    lib.aqshade_mesh.argtypes = [P, P, I, P, I, I, P, P, P, P]
    lib.aqshade_trace.argtypes = [P, P, I, P, I, I, P, P, P]
    lib.aqshade_container.argtypes = [P, P, I, P, I, I, P, P]
    rng = np.random.default_rng(2024)
    sky = rng.integers(0, 256, (6, 16, 16, 3), dtype=np.uint8)
    logo = rng.integers(0, 256, (12, 20, 3), dtype=np.uint8)
    res = {"sky": sky, "logo": logo, "windows": np.array(SHADE_WINDOWS, np.float32)}
    views, projs, eyes = [], [], []
    for w, h, size in SHADE_WINDOWS:
        v, p, e = np.zeros(16, np.float32), np.zeros(16, np.float32), np.zeros(3, np.float32)
        lib.aqshade_camera(int(w), int(h), float(size), v.ctypes.data, p.ctypes.data, e.ctypes.data)
        views.append(v); projs.append(p); eyes.append(e)
    res.update(cam_view=np.array(views), cam_projection=np.array(projs), cam_eye=np.array(eyes))
    dc = RenderOracle.draw_command_default(320, 160, 10.0, 32)
    n = 128
    mesh_in, mesh_out, trace_in, trace_out, cont_in, cont_out = [], [], [], [], [], []
    for env in range(3):
        dc.environment_mode = env
        for mode in range(8):
            dc.render_mode = mode
            for _ in range(n):
                pos = rng.uniform(-2, 12, 3).astype(np.float32)
                nrm = rng.normal(size=3).astype(np.float32)
                tex = (rng.uniform(0, 60, 4) * (rng.random(4) < 0.7)).astype(np.float32)
                out = np.zeros(4, np.float32)
                lib.aqshade_mesh(ct.addressof(dc), sky.ctypes.data, 16, logo.ctypes.data, 20, 12, pos.ctypes.data,
                                 nrm.ctypes.data, tex.ctypes.data, out.ctypes.data)
                mesh_in.append(np.concatenate([[env, mode], pos, nrm, tex]).astype(np.float32))
                mesh_out.append(out)
        for k in range(4 * n):
            org = rng.uniform(-10, 20, 3).astype(np.float32)
            d = rng.normal(size=3).astype(np.float32)
            if k % 7 == 0:
                d[rng.integers(3)] = 0
            out = np.zeros(4, np.float32)
            lib.aqshade_trace(ct.addressof(dc), sky.ctypes.data, 16, logo.ctypes.data, 20, 12, org.ctypes.data,
                              d.ctypes.data, out.ctypes.data)
            trace_in.append(np.concatenate([[env], org, d]).astype(np.float32))
            trace_out.append(out)
        for _ in range(n):
            pos = rng.uniform(-15, 25, 3).astype(np.float32)
            out = np.zeros(4, np.float32)
            lib.aqshade_container(ct.addressof(dc), sky.ctypes.data, 16, logo.ctypes.data, 20, 12, pos.ctypes.data,
                                  out.ctypes.data)
            cont_in.append(np.concatenate([[env], pos]).astype(np.float32))
            cont_out.append(out)
    res.update(mesh_in=np.array(mesh_in), mesh_out=np.array(mesh_out), trace_in=np.array(trace_in),
               trace_out=np.array(trace_out), container_in=np.array(cont_in), container_out=np.array(cont_out))
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE))
    ap.add_argument("--only", choices=["all", "ink", "mesh", "sph", "shade"], default="all")
    a = ap.parse_args()
    out = pathlib.Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    if a.only in ("all", "mesh"):
        np.savez_compressed(out / "texture_linear_probe.npz", **record_linear_probe())
        np.savez_compressed(out / "ref_mesh.npz", **record_mesh())
        print("mesh fixtures recorded")
    if a.only in ("all", "sph"):
        np.savez_compressed(out / "ref_sph.npz", **record_sph())
        print("sph fixtures recorded")
    if a.only in ("all", "shade"):
        np.savez_compressed(out / "ref_shade.npz", **record_shade())
        print("shade fixtures recorded")
    if a.only in ("all", "ink"):
        np.savez_compressed(out / "ref_ink.npz", **record_ink())
        print("ink fixtures recorded")
    if a.only != "all":
        return
    probe = texture_probe()
    (out / "texture_probe.json").write_text(json.dumps(probe, indent=1))
    print("texture probe:", {k: v for k, v in probe.items() if k != "reads"})
    spreads = {}
    for name, steps in GOLDEN_SCENES.items():
        data, spread = record_scene(name, steps)
        np.savez_compressed(out / f"ref_{name}.npz", **data)
        spreads[name] = spread
        print(name, "recorded", len(data), "arrays; max float spread",
              max([v for k, v in spread.items() if isinstance(v, float)] + [0.0]))
    (out / "reference_spread.json").write_text(json.dumps(spreads, indent=1, sort_keys=True))
    np.savez_compressed(out / "ref_special.npz", **record_special())
    print("special fixtures recorded")


if __name__ == "__main__":
    main()
