"""Benchmark of the B200 FLIP step on the 128^3 ball-drop workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the configuration the headline metric is quoted on): 128^3 MAC grid,
domain 10, pool y < 0.3 plus a sphere r = 0.12 at (0.5, 0.7, 0.5), 8 jittered
particles per fluid cell (5.23M particles, seeded rand() sequence), dt 0.005,
FLIP 0.95, gravity (0,-9.8,0), zero initial pressure each step, Jacobi run to
relative residual 1e-4 (FP64, checked every 40 sweeps), capped at 2000 sweeps.
A step is one simulationStep of that scene; its per-step working set
(particle state ~250 MB plus grids) exceeds the 126 MB L2, so no flush is
needed between steps.

One JSON line on rank 0.  With N > 1 (torchrun) each rank steps its own
replica of the scene (the path has no data exchange): weak scaling, time =
max over ranks.  `--impl reference` times the CPU restatement of the
reference step (oracle/, the reference has no CPU implementation of its own)
on the host cores, on rank 0 only.

`--workload batch` measures the batch of independent scenes instead: 256
ball-drop scenes whose sizes are drawn per axis from {24, 32, 48, 64}
(seeded), pool depth 0.1-0.4 plus 1-2 spheres r 0.08-0.2, 8 particles per
fluid cell (~40M particles), dt 0.01, zero-init Jacobi to relative residual
1e-4 per scene (cap 2000); a step advances every scene once, and the value is
batch steps/s.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "FLIP steps/s at 128^3 x 8ppc, Jacobi to relative residual 1e-4 (plain, zero-init)"
UNIT = "steps/s"
MEASURED_PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
JACOBI_BYTES_PER_CELL = 13  # p read 4 + p write 4 + rhs 4 + cell type 1
BATCH_METRIC = ("batch steps/s, 256 independent scenes of sizes {24,32,48,64} per axis x 8ppc, "
                "Jacobi to relative residual 1e-4 per scene (plain, zero-init)")
BATCH_SEED = 2024


def workload_config(size=128, pressure_init="zero"):
    from aquarius_b200 import _abi
    vols = [dict(shape="box", min=(0, 0, 0), max=(1, 0.3, 1), phase=0),
            dict(shape="sphere", center=(0.5, 0.7, 0.5), radius=0.12, phase=0)]
    return _abi.make_config(
        (size, size, size), vols, timestep=0.005, flip_coeff=0.95, particle_jitter=0.05,
        pressure_init=_abi.PRESSURE_ZERO if pressure_init == "zero" else _abi.PRESSURE_CARRY,
        solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=1e-4, max_iterations=2000, check_interval=40)


def config1_config():
    """50^3 ball drop, pool y < 0.2 plus a sphere r 0.15 at
    (0.5, 0.65, 0.5), 8 particles per cell, dt 0.01, FLIP 0.95, 100 Jacobi
    sweeps per step with the pressure carried as the reference does."""
    from aquarius_b200 import _abi
    vols = [dict(shape="box", min=(0, 0, 0), max=(1, 0.2, 1), phase=0),
            dict(shape="sphere", center=(0.5, 0.65, 0.5), radius=0.15, phase=0)]
    return _abi.make_config((50, 50, 50), vols, timestep=0.01, flip_coeff=0.95, particle_jitter=0.05,
                            pressure_init=_abi.PRESSURE_CARRY, solve_mode=_abi.SOLVE_FIXED, pressure_iterations=100)


def config_desc(size, pressure_init):
    return {"workload": f"ball drop {size}^3 x 8ppc (pool y<0.3 + sphere r=0.12), dt=0.005, "
                        f"Jacobi to rel-res 1e-4 cap 2000, {pressure_init}-init pressure",
            "grid": [size, size, size], "particles_per_cell": 8, "pressure_init": pressure_init,
            "l2": "per-step working set > 126 MB L2 (no flush needed)"}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def reduce_max(x: float, dist, device: str) -> float:
    """Max of a per-rank scalar over all ranks (identity without a process group)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_value(steps_per_rank: int, world: int, max_ms: float) -> float:
    """Whole-job steps/s: every rank steps its own replica; time = slowest rank."""
    return world * steps_per_rank / (max_ms / 1000.0)


def jacobi_kernel_name(f) -> str:
    return jacobi_kernel_name_of(f.jacobi_plan())


def jacobi_kernel_name_of(plan) -> str:
    levels, rows, xplanes = plan
    if rows == 1:
        return "k_persist_solve (whole solve in one cooperative launch)"
    if rows == 0:
        return f"k_jacobi_flat<{xplanes}> (1 sweep/launch, float4 z-quads)"
    if rows == 3:
        return "k_jacobi_list (1 sweep/launch over the listed active warp rows, one resident wave)"
    if rows == 4:
        shapes = ["8x40x24", "16x24x24", "8x32x24", "16x16x24", "8x16x24", "24x16x24", "8x48x24"]
        return (f"k_resident_solve<tiles {shapes[xplanes]}, halo {levels}> (whole solve in one cooperative launch, "
                f"tiles resident in shared memory, halos exchanged every {levels} sweeps)")
    if rows == 2:
        return f"k_jacobi_cube<{levels} sweeps/launch, {xplanes}x{xplanes}x{32 - 2 * levels} tiles> (shared-memory cubes)"
    return f"k_jacobi<{levels} sweeps/launch, {rows} rows, {xplanes} x-planes> (temporally blocked)"


def measured_traffic(f):
    """DRAM bytes per launch of the dominant kernel from the committed ncu
    summary (profiles/roofline_traffic.json), when it covers this kernel."""
    try:
        d = json.loads((ROOT / "profiles" / "roofline_traffic.json").read_text())
        levels, rows, xplanes = f.jacobi_plan()
        key = {(0, 1): "k_jacobi_flat", (3, 1): "k_jacobi_list"}.get((rows, xplanes))
        if rows == 4:
            key = f"k_resident_solve/{levels}/{xplanes}"
        if key in d:
            return d[key]["bytes_per_launch"]
    except Exception:
        pass
    return None


def batch_traffic(cells: int):
    """DRAM bytes per batched sweep: the per-updated-cell traffic of the
    committed 32-scene capture (profiles/roofline_traffic.json) x cells."""
    try:
        d = json.loads((ROOT / "profiles" / "roofline_traffic.json").read_text())
        return d["kb_jacobi_rows"]["bytes_per_updated_cell"] * cells
    except Exception:
        return None


def measured_hbm_peak():
    try:
        d = json.loads(MEASURED_PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def cpu_baseline_sample(size: int, pressure_init: str, steps: int = 1) -> dict:
    """Times the CPU oracle on `steps` full steps of the same workload."""
    sys.path.insert(0, str(ROOT / "tests"))
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    import oracle_binding  # test infrastructure: the CPU restatement of the reference step
    cfg = workload_config(size, pressure_init)
    t0 = time.perf_counter()
    o = oracle_binding.Oracle(cfg)
    t_init = time.perf_counter() - t0
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    st = o.solve_stats()
    o.close()
    return {"value": steps / dt, "unit": UNIT, "cores": oracle_binding.oracle_threads(), "kind": "port",
            "sample": f"{steps} full step(s) of the {size}^3 workload on the OpenMP oracle "
                      f"(init {t_init:.1f}s excluded; last solve {st['iterations']} sweeps)",
            "seconds": dt}


def batch_cpu_sample(cfgs, budget_s: float = 20.0) -> dict:
    """One step of as many scenes as fit in the budget on the CPU oracle
    (scene init excluded), extrapolated to the whole batch by cell count."""
    sys.path.insert(0, str(ROOT / "tests"))
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    import oracle_binding  # test infrastructure: the CPU restatement of the reference step
    total_cells = sum(c.size_x * c.size_y * c.size_z for c in cfgs)
    spent, cells, done = 0.0, 0, 0
    for c in cfgs:
        o = oracle_binding.Oracle(c)
        t0 = time.perf_counter()
        o.step(1)
        spent += time.perf_counter() - t0
        o.close()
        cells += c.size_x * c.size_y * c.size_z
        done += 1
        if spent > budget_s:
            break
    est = spent * total_cells / cells
    return {"value": 1.0 / est, "unit": UNIT, "cores": oracle_binding.oracle_threads(), "kind": "port",
            "sample": f"one step of scenes 0..{done - 1} ({cells} of {total_cells} cells) on the OpenMP oracle, "
                      f"{spent:.1f}s, extrapolated to the batch by cell count", "seconds": spent}


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    if args.workload == "batch":
        from aquarius_b200.scenes import batch_configs, batch_desc
        cfgs = batch_configs(args.scenes, seed=BATCH_SEED)
        cb = batch_cpu_sample(cfgs, budget_s=min(150.0, 20.0 * max(1, args.steps)))
        v = cb["value"]
        line = {"impl": "reference", "metric": BATCH_METRIC, "value": v, "unit": UNIT, "n_gpus": world,
                "steps": 1, "warmup": 0, "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": batch_desc(args.scenes, BATCH_SEED)},
                "cpu_baseline": dict(cb), "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                                                  "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    # each timed step is one full CPU step of the workload; warm-up steps are
    # bounded to one, and timed steps to what fits in a few minutes
    sys.path.insert(0, str(ROOT / "tests"))
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    import oracle_binding
    cfg = workload_config(args.size, args.pressure_init)
    o = oracle_binding.Oracle(cfg)
    o.step(min(args.warmup, 10))
    budget_s = 150.0
    done, t0 = 0, time.perf_counter()
    while done < args.steps:
        o.step(1)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    v = done / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": done,
            "warmup": min(args.warmup, 10), "ms_per_step": 1000 * dt / done, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_desc(args.size, args.pressure_init),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": oracle_binding.oracle_threads(), "kind": "port",
                             "sample": f"{done} full CPU step(s) of the workload, OpenMP restatement of the "
                                       f"reference step (the reference has no CPU path)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, dist):
    import numpy as np
    import torch

    import aquarius_b200 as aq

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    cfg = workload_config(args.size, args.pressure_init)
    cfg.device = dev
    f = aq.Fluid(cfg)
    if args.eager:
        f.set_graph_mode(False)
    stream = torch.cuda.ExternalStream(f.stream(), device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return reduce_max(x, dist, f"cuda:{dev}")

    # warm-up (builds and instantiates the step graph); the Jacobi plan is
    # tuned on the warmed-up system, then the graph is rebuilt and warmed again
    f.step(args.warmup)
    f.synchronize()
    tune = f.autotune(200) if not args.no_tune else {"plan": f.jacobi_plan(), "sweep_us": None}
    f.step(1)
    f.synchronize()
    st0 = f.solve_stats()
    per_step, per_block = f.launch_counts()

    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.4)
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        f.step(args.steps)
        ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms)
    st1 = f.solve_stats()
    sweeps = st1["total_sweeps"] - st0["total_sweeps"]
    blocks = st1["total_blocks"] - st0["total_blocks"]
    launches = args.steps * per_step + blocks * per_block
    value = weak_scaling_value(args.steps, world, ms_max)

    # e2e: the same steps through the C-ABI host-buffer entry point; every step
    # uploads the particle state from pinned host memory and reads it back
    n = f.particleCount
    pin_pos = torch.empty((3, n), dtype=torch.float32).pin_memory()
    pin_vel = torch.empty((3, n), dtype=torch.float32).pin_memory()
    pos_np, vel_np = pin_pos.numpy(), pin_vel.numpy()
    f.step_host(0, None, None, pos_np, vel_np)
    e2e_steps = max(1, min(args.steps, 10))
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            f.step_host(1, pos_np, vel_np, pos_np, vel_np)
        e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_wall = time.perf_counter() - t0
    e2e_value = weak_scaling_value(e2e_steps, world, e2e_ms)

    # roofline of the dominant kernel: Jacobi sweeps on the last step's system
    hbm_peak, peak_kind = measured_hbm_peak()
    jb = f.benchmark_pressure(400)
    sweep_ms = jb["ms"] / 400
    cells = jb["cells_per_sweep"]
    achieved_gbs = JACOBI_BYTES_PER_CELL * cells / (sweep_ms / 1000.0) / 1e9
    C = args.size ** 3
    full_gbs = JACOBI_BYTES_PER_CELL * C / (sweep_ms / 1000.0) / 1e9

    # pressure error of the plain solve against FP64 PCG on the same system
    f.step(1)
    pstats = f.solve_stats()
    pcg = f.pcg_reference(rel_tol=1e-12, max_iter=200000)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": dict(config_desc(args.size, args.pressure_init), launch="kernel-by-kernel" if args.eager
                       else "one CUDA graph per step"),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 2 * 12 * n,
                "d2h_bytes_per_step": 2 * 12 * n, "steps": e2e_steps, "wall_s": e2e_wall,
                "path": "aq_fluid_step_host (C ABI), pinned host particle state in and out every step"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": jacobi_kernel_name(f), "achieved": achieved_gbs,
                     "peak": hbm_peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved_gbs / hbm_peak,
                     "traffic": measured_traffic(f),
                     "algorithmic_bytes": f"{JACOBI_BYTES_PER_CELL} B per updated cell per sweep x {cells} cells",
                     "sweep_us": sweep_ms * 1000.0, "full_domain_equiv_gbs": full_gbs},
        "clocks": clk,
        "solver": {"sweeps_per_step": sweeps / args.steps, "blocks_per_step": blocks / args.steps,
                   "last_rel_residual": pstats["rel_residual"], "last_iterations": pstats["iterations"],
                   "converged": pstats["converged"], "fluid_cells": pstats["fluid_cells"],
                   "pressure_rel_error_vs_fp64_pcg": pcg["rel_error"], "pcg_iterations": pcg["iterations"]},
        "particles": n,
        "jacobi_plan": {"levels": tune["plan"][0], "rows": tune["plan"][1], "x_planes": tune["plan"][2],
                        "tuned_sweep_us": tune["sweep_us"]},
    }
    line["mesh"] = mesh_timing(f, stream)
    line["render"] = render_timing(f, args.size)
    plain_rel = [st1["rel_residual"], pstats["rel_residual"]]
    plan = f.jacobi_plan()
    f.close()
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        line["reference_gpu"] = reference_gpu_comparator(args, dev, plan)
    if not args.no_learned:
        line["learned"] = learned_arm(args, dev, stream, max(plain_rel), ms_max / args.steps, dist, plan)
        alt = ROOT / "aquarius_b200" / "weights" / f"unet_{args.size}_from64.bin"
        if alt.exists():  # the 64^3 network with a recalibrated output scale, no training at this size
            line["learned_from64"] = learned_arm(args, dev, stream, max(plain_rel), ms_max / args.steps, dist,
                                                 plan, wpath=alt)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(args.size, args.pressure_init, steps=1)
    if rank == 0:
        print(json.dumps(line), flush=True)


def mesh_timing(f, stream, reps: int = 10) -> dict:
    """The surface mesher (Mesher::mesh) on the workload's particles after
    its steps: SDF on the h/2 grid and marching cubes on the 128^3 grid into
    a device buffer, timed with CUDA events on the fluid's stream over reps
    calls (each call ends with a host read of the cube count)."""
    import torch

    info = f.mesh_info()
    cap = 1 << 19
    buf = torch.empty((cap * 90,), dtype=torch.float32, device="cuda")
    cubes = 0
    for _ in range(2):
        cubes = f.mesh_into(buf.data_ptr(), cap)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(reps):
            f.mesh_into(buf.data_ptr(), cap)
        e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    vertices = int((buf[: cubes * 90].view(cubes, 15, 6).abs().sum(dim=2) != 0).sum().item())
    del buf
    return {"ms_per_mesh": ms, "cubes": cubes, "triangles": vertices // 3, "sdf_grid": list(info["sdf"]),
            "mesh_grid": list(info["mesh"]), "reps": reps,
            "path": "aq_fluid_mesh into a device buffer (the reference's VBO layout)"}


def render_timing(f, size: int, reps: int = 10, width: int = 1728, height: int = 864) -> dict:
    """The headless frame of the reference's renderer (main.cu's first frame:
    skybox, container floor, phase-thickness sprites, the fluid mesh shaded
    with reflection/refraction) on the workload's particles, in the window
    main.cu opens on a 1920-wide screen.  Fluid::draw as aq_fluid_draw (mesh +
    point VBO + frame) and the frame alone (aq_renderer_draw from resident
    VBOs), host wall clock per call with a synchronize after each (the draw
    reads its primitive-tile pair counts back to the host once per frame)."""
    import time

    import numpy as np
    import torch

    import aquarius_b200 as aq
    rng = np.random.default_rng(11)
    r = aq.Renderer(torch.cuda.current_device())
    r.set_skybox(rng.integers(0, 256, (6, 256, 256, 3), dtype=np.uint8))
    dc = aq.draw_command_default(width, height, f.getContainerSize(), size)
    img = torch.empty((height * width * 4,), dtype=torch.uint8, device="cuda")

    def best(fn):
        for _ in range(2):
            fn()
        r.synchronize()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            r.synchronize()
            ts.append(time.perf_counter() - t0)
        return 1e3 * float(np.median(ts))

    full_ms = best(lambda: f.draw(dc, r, img.data_ptr()))
    recs = f.download_mesh()
    mesh = torch.from_numpy(np.ascontiguousarray(recs.reshape(-1, 6))).cuda()
    pts = torch.empty((f.particleCount * 7,), dtype=torch.float32, device="cuda")
    f.points_vbo_into(pts.data_ptr())
    torch.cuda.synchronize()
    frame_ms = best(lambda: r.draw(dc, pts.data_ptr(), f.particleCount, mesh.data_ptr(), mesh.shape[0],
                                   img.data_ptr()))
    out = {"ms_per_frame": frame_ms, "ms_per_fluid_draw": full_ms, "window": [width, height],
           "render_mode": "multiphase mesh", "environment": "skybox", "particles": f.particleCount,
           "mesh_vertices": int(mesh.shape[0]), "launches": r.launches(), "reps": reps,
           "path": "aq_renderer_draw (frame from resident VBOs) / aq_fluid_draw (Fluid::draw)",
           "reference": "unavailable on this box (GL)"}
    r.close()
    return out


def reference_gpu_step_ms(size: int, steps: int = 5, workload: str = "ball128") -> dict:
    """Milliseconds per simulationStep of the reference's own kernels on the
    fixed-sweep comparator workload.  Runs in a process of its own: the
    reference's init sets the device's printf FIFO size
    (Fluid/Fluid_3D_FLIP.cu:489), which CUDA refuses once other kernels ran
    in the context."""
    from aquarius_b200 import _abi
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_binding
    if workload == "ball50":
        cfg = config1_config()
    else:
        cfg = workload_config(size, "carry")
        cfg.solve_mode = _abi.SOLVE_FIXED
        cfg.pressure_iterations = 2000
    ref = oracle_binding.RefFluid(cfg)
    ref.step(2)
    ms = min(ref.time_steps(steps) for _ in range(3)) / steps
    ref.close()
    return {"reference_ms_per_step": ms}


def reference_gpu_comparator(args, dev, plan, steps: int = 5) -> dict:
    """The reference's own FLIP kernels (Fluid_3D_FLIP::Fluid compiled headless
    from its sources into oracle/_ref/libaqref.so, Fluid/Fluid_3D_FLIP.cu:316-352)
    on this workload with the reference's fixed-iteration Jacobi (2000
    sweeps; pressure carried across steps as the reference does,
    Fluid/Fluid_3D_common.cu:48-55), timed with CUDA events on the legacy
    default stream it launches on (its own device synchronisations inside a
    step included), beside this library on the same scene, the same 2000
    sweeps (AQ_SOLVE_FIXED, carried pressure) and the tuned Jacobi plan, timed
    on the fluid's stream.  Not the product path: the comparator the plain
    step is measured against."""
    import torch

    import aquarius_b200 as aq
    from aquarius_b200 import _abi
    if not (ROOT / "oracle" / "_ref" / "libaqref.so").exists():
        return {"unavailable": "the headless reference build (oracle/_ref/libaqref.so) is not present"}
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(dev)))
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--reference-gpu-only", "--size", str(args.size)],
                       capture_output=True, text=True, env=env, timeout=600)
    try:
        ref = json.loads(r.stdout.strip().splitlines()[-1])
    except Exception:
        return {"unavailable": f"reference run failed: {(r.stderr or r.stdout)[-300:]}"}
    cfg = workload_config(args.size, "carry")
    cfg.solve_mode = _abi.SOLVE_FIXED
    cfg.pressure_iterations = 2000
    cfg.device = dev
    f = aq.Fluid(cfg)
    if plan[1] != 1:
        f.set_jacobi_plan(*plan)
    f.step(3)
    f.synchronize()
    st = torch.cuda.ExternalStream(f.stream(), device=dev)
    lib = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        f.step(steps)
        e1.record(st)
        e1.synchronize()
        lib.append(e0.elapsed_time(e1) / steps)
    sweeps = f.solve_stats()["iterations"]
    f.close()
    lib_ms = min(lib)
    ref_ms = ref["reference_ms_per_step"]
    return {"workload": f"{args.size}^3 ball drop, 2000 fixed Jacobi sweeps per step, carried pressure",
            "reference_ms_per_step": ref_ms, "library_ms_per_step": lib_ms, "library_sweeps_per_step": sweeps,
            "speedup": ref_ms / lib_ms, "library_jacobi_plan": list(plan),
            "reference_build": "Fluid/*.cu compiled headless with the reference's flags (-use_fast_math) for sm_100a"}


def learned_arm(args, dev, stream, plain_residual: float, plain_ms: float, dist, plan, wpath=None) -> dict:
    """The same workload with the learned warm start (AQ_PRESSURE_LEARNED) and
    the plain step's Jacobi plan: (a) to the same target 1e-4 (cap 2000), (b)
    to the residual the plain step reached at its cap, i.e. at equal achieved
    residual.  wpath: the network (default weights/unet_<size>.bin)."""
    import torch

    import aquarius_b200 as aq
    from aquarius_b200 import _abi
    if wpath is None:
        wpath = ROOT / "aquarius_b200" / "weights" / f"unet_{args.size}.bin"
    if not wpath.exists():
        return {"unavailable": f"no trained weights for {args.size}^3 ({wpath.name})"}
    net = aq.UNet(device=dev, weights=wpath)
    out = {"weights": wpath.name, "parameters": net.parameter_count(), "jacobi_plan": list(plan)}
    for name, target in (("to_1e-4", 1e-4), ("to_plain_residual", plain_residual)):
        cfg = workload_config(args.size, "zero")
        cfg.pressure_init = _abi.PRESSURE_LEARNED
        cfg.rel_residual = float(target)
        cfg.device = dev
        f = aq.Fluid(cfg)
        if plan[1] != 1:  # the persistent solve does not take the warm start
            f.set_jacobi_plan(*plan)
        f.set_warm_start(net)
        f.step(args.warmup)
        f.synchronize()
        s0 = f.solve_stats()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        lstream = torch.cuda.ExternalStream(f.stream(), device=dev)
        with torch.cuda.stream(lstream):
            ev0.record(lstream)
            f.step(args.steps)
            ev1.record(lstream)
        ev1.synchronize()
        ms = reduce_max(ev0.elapsed_time(ev1), dist, f"cuda:{dev}") / args.steps
        s1 = f.solve_stats()
        f.step(1)
        s2 = f.solve_stats()
        pcg = f.pcg_reference(rel_tol=1e-12, max_iter=200000)
        out[name] = {"target_rel_residual": target, "steps_per_s": 1000.0 / ms, "ms_per_step": ms,
                     "time_vs_plain": ms / plain_ms,
                     "sweeps_per_step": (s1["total_sweeps"] - s0["total_sweeps"]) / args.steps,
                     "last_rel_residual": s2["rel_residual"], "last_iterations": s2["iterations"],
                     "converged": s2["converged"], "warm_start_kept": s2["warm_start"] == 1,
                     "residual_after_20_sweeps": {"learned": s2["warm_rel_residual"],
                                                  "zero_init": s2["zero_rel_residual"]},
                     "pressure_rel_error_vs_fp64_pcg": pcg["rel_error"]}
        f.close()
    net.close()
    return out


def run_config1(args, rank: int, world: int, dist):
    """BASELINE config 1 (the reference's own scale: 50^3, 100 Jacobi sweeps):
    steps/s of this library (graph), end to end through the host-buffer
    C-ABI step, of the reference's own kernels on the same GPU (child
    process, CUDA events) and of the CPU oracle.  50 is not a multiple of 4,
    so the library runs its tiled sweep kernels here."""
    import torch

    import aquarius_b200 as aq
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    cfg = config1_config()
    cfg.device = dev
    f = aq.Fluid(cfg)
    stream = torch.cuda.ExternalStream(f.stream(), device=dev)
    f.step(args.warmup)
    f.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.3)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    f.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    ms = reduce_max(e0.elapsed_time(e1), dist, f"cuda:{dev}")
    value = weak_scaling_value(args.steps, world, ms)
    n = f.particleCount
    pin_pos = torch.empty((3, n), dtype=torch.float32).pin_memory().numpy()
    pin_vel = torch.empty((3, n), dtype=torch.float32).pin_memory().numpy()
    f.step_host(0, None, None, pin_pos, pin_vel)
    e0.record(stream)
    for _ in range(args.steps):
        f.step_host(1, pin_pos, pin_vel, pin_pos, pin_vel)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = reduce_max(e0.elapsed_time(e1), dist, f"cuda:{dev}")
    hbm_peak, peak_kind = measured_hbm_peak()
    jb = f.benchmark_pressure(400)
    sweep_ms = jb["ms"] / 400
    cells = jb["cells_per_sweep"]
    achieved = JACOBI_BYTES_PER_CELL * cells / (sweep_ms / 1000.0) / 1e9
    plan = f.jacobi_plan()
    f.close()
    line = {"metric": "FLIP steps/s at 50^3 x 8ppc, 100 Jacobi sweeps per step (BASELINE config 1)",
            "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": "ball drop 50^3 x 8ppc (pool y<0.2 + sphere r=0.15), dt=0.01, 100 Jacobi "
                                   "sweeps, carried pressure", "grid": [50, 50, 50], "particles_per_cell": 8,
                       "l2": "working set < L2 (the reference's own scale); no flush"},
            "e2e": {"value": weak_scaling_value(args.steps, world, e2e_ms), "unit": UNIT,
                    "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 24 * n,
                    "path": "aq_fluid_step_host (C ABI), pinned host particle state in and out every step"},
            "roofline": {"bound": "hbm", "kernel": jacobi_kernel_name_of(plan), "achieved": achieved,
                         "peak": hbm_peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm_peak,
                         "traffic": None, "sweep_us": sweep_ms * 1000.0,
                         "algorithmic_bytes": f"{JACOBI_BYTES_PER_CELL} B per updated cell per sweep x {cells} cells"},
            "clocks": clk, "particles": n}
    if rank == 0 and world == 1:
        env = dict(os.environ)
        r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--reference-gpu-only", "--workload", "ball50"],
                           capture_output=True, text=True, env=env, timeout=600)
        try:
            ref_ms = json.loads(r.stdout.strip().splitlines()[-1])["reference_ms_per_step"]
            line["reference_gpu"] = {"reference_ms_per_step": ref_ms, "library_ms_per_step": ms / args.steps,
                                     "speedup": ref_ms / (ms / args.steps)}
        except Exception:
            line["reference_gpu"] = {"unavailable": (r.stderr or r.stdout)[-300:]}
        if not args.no_cpu_baseline:
            sys.path.insert(0, str(ROOT / "tests"))
            import oracle_binding
            o = oracle_binding.Oracle(config1_config())
            o.step(1)
            t0 = time.perf_counter()
            k = 0
            while k < 20 and time.perf_counter() - t0 < 15.0:
                o.step(1)
                k += 1
            dt = time.perf_counter() - t0
            o.close()
            line["cpu_baseline"] = {"value": k / dt, "unit": UNIT, "cores": oracle_binding.oracle_threads(),
                                    "kind": "port", "sample": f"{k} steps of the same scene on the OpenMP oracle"}
        print(json.dumps(line), flush=True)


def run_batch(args, rank: int, world: int, dist):
    import torch

    import aquarius_b200 as aq
    from aquarius_b200.scenes import batch_configs, batch_desc

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    # every rank steps its own batch (weak scaling); ranks draw different scene sets
    cfgs = batch_configs(args.scenes, seed=BATCH_SEED + rank, device=dev)
    t0 = time.perf_counter()
    b = aq.Batch(cfgs)
    t_init = time.perf_counter() - t0
    tot = b.totals()
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    b.step(args.warmup)
    b.synchronize()
    if args.no_tune:
        xp, pipe = b.sweep_plan()
        tune = {"x_planes": xp, "pipelined": pipe, "sweep_us": None}
    else:
        tune = b.autotune(50)
    b.step(1)
    b.synchronize()
    per_step, per_block = b.launch_counts()
    s0 = [b.solve_stats(i) for i in range(b.scene_count)]

    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.4)
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        b.step(args.steps)
        ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    ms_max = reduce_max(ms, dist, f"cuda:{dev}")
    s1 = [b.solve_stats(i) for i in range(b.scene_count)]
    # the solve loop runs until its slowest scene stops: loop blocks = max over scenes
    loop_blocks = max(x["total_blocks"] - y["total_blocks"] for x, y in zip(s1, s0))
    launches = args.steps * per_step + loop_blocks * per_block
    value = weak_scaling_value(args.steps, world, ms_max)
    sweeps = [x["total_sweeps"] - y["total_sweeps"] for x, y in zip(s1, s0)]
    conv = sum(1 for x in s1 if x["converged"])

    # e2e through the host-buffer entry point: all particle state in and out
    n = tot["particles"]
    pin_pos = torch.empty((3, n), dtype=torch.float32).pin_memory()
    pin_vel = torch.empty((3, n), dtype=torch.float32).pin_memory()
    pos_np, vel_np = pin_pos.numpy(), pin_vel.numpy()
    b.step_host(0, None, None, pos_np, vel_np)
    e2e_steps = max(1, min(args.steps, 5))
    barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            b.step_host(1, pos_np, vel_np, pos_np, vel_np)
        e1.record(stream)
    e1.synchronize()
    e2e_ms = reduce_max(e0.elapsed_time(e1), dist, f"cuda:{dev}")

    hbm_peak, peak_kind = measured_hbm_peak()
    jb = b.benchmark_pressure(200)
    sweep_ms = jb["ms"] / 200
    cells = jb["cells_per_sweep"]
    achieved = JACOBI_BYTES_PER_CELL * cells / (sweep_ms / 1000.0) / 1e9
    line = {
        "metric": BATCH_METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": batch_desc(args.scenes, BATCH_SEED), "scenes": b.scene_count,
                   "cells": tot["cells"], "particles": n, "launch": "one CUDA graph per step, one launch per stage",
                   "l2": "per-step working set > 126 MB L2 (no flush needed)", "init_s": t_init},
        "scene_steps_per_s": value * b.scene_count,
        "e2e": {"value": weak_scaling_value(e2e_steps, world, e2e_ms), "unit": UNIT,
                "h2d_bytes_per_step": 2 * 12 * n, "d2h_bytes_per_step": 2 * 12 * n, "steps": e2e_steps,
                "path": "aq_batch_step_host (C ABI), pinned host particle state of all scenes in and out"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": f"kb_jacobi_rows<{tune['x_planes']}, {'pipelined' if tune['pipelined'] else 'plain'}> "
                               "(one sweep of every live scene per launch, packed rows)",
                     "achieved": achieved, "peak": hbm_peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": batch_traffic(cells),
                     "algorithmic_bytes": f"{JACOBI_BYTES_PER_CELL} B per updated cell per sweep x {cells} cells",
                     "sweep_us": sweep_ms * 1000.0},
        "clocks": clk,
        "solver": {"mean_sweeps_per_scene_step": sum(sweeps) / len(sweeps) / args.steps,
                   "max_sweeps_per_scene_step": max(sweeps) / args.steps,
                   "loop_blocks_per_step": loop_blocks / args.steps,
                   "scenes_converged_last_step": conv},
        "sweep_plan": {"x_planes_per_item": tune["x_planes"], "pipelined": tune["pipelined"],
                       "tuned_sweep_us": tune["sweep_us"]},
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = batch_cpu_sample(cfgs)
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()


def sph_cpu_sample(cfg, budget_s: float = 15.0) -> dict:
    """The CPU oracle stepping the same solver on the host cores, on a
    smaller particle budget (a bounded sample); steps/s scaled to the
    workload's particle count (per-particle cost is constant)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_binding import SphOracle, oracle_threads
    from aquarius_b200 import _abi
    import ctypes as ct
    small = _abi.SphConfig()
    ct.memmove(ct.byref(small), ct.byref(cfg), ct.sizeof(cfg))
    small.max_particle_count = 300000
    small.stream = None
    o = SphOracle(small)
    t0 = time.perf_counter()
    steps = 0
    while time.perf_counter() - t0 < budget_s and steps < 50:
        o.step(1)
        steps += 1
    dt = time.perf_counter() - t0
    o.close()
    return {"particles": o.n, "steps": steps, "seconds": dt, "threads": oracle_threads()}


def run_sph(args, rank: int, world: int, dist):
    """The reference's particle-only solvers (PBF or PCISPH, reference
    defaults otherwise) with a particle budget of args.particles (default
    3e7: about 5.6M particles in the default pool + ball scene), one CUDA
    graph per step.  Reports steps/s; the e2e arm uploads positions and
    velocities from pinned host memory, steps and downloads positions."""
    import ctypes as ct

    import numpy as np
    import torch

    import aquarius_b200 as aq
    from aquarius_b200 import _abi
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    method = _abi.SPH_PBF if args.workload == "pbf" else _abi.SPH_PCISPH
    stream = torch.cuda.Stream(device=dev)
    cfg = _abi.sph_config(method, max_particle_count=int(args.particles), device=dev)
    cfg.stream = stream.cuda_stream
    t0 = time.perf_counter()
    s = aq.Sph(cfg)
    t_init = time.perf_counter() - t0
    s.step(args.warmup)
    s.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.4)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    s.step(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clk = clocks.stop()
    ms = reduce_max(ev0.elapsed_time(ev1), dist, f"cuda:{dev}")
    value = weak_scaling_value(args.steps, world, ms)
    # e2e: state in from pinned host buffers, one step, positions out
    n = s.n
    pin_p = torch.empty((3, n), dtype=torch.float32).pin_memory()
    pin_v = torch.empty((3, n), dtype=torch.float32).pin_memory()
    st0 = s.get_state(["position", "velocity"])
    pin_p.numpy()[:] = st0["position"]
    pin_v.numpy()[:] = st0["velocity"]
    e2e_steps = max(1, min(args.steps, 5))
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(e2e_steps):
        sst = _abi.make_sph_state(n, {"position": pin_p.numpy(), "velocity": pin_v.numpy()})
        aq._check(s._lib.aq_sph_upload_state(s._h, ct.byref(sst)))
        s.step(1)
        out = _abi.make_sph_state(n, {"position": pin_p.numpy()})
        aq._check(s._lib.aq_sph_download_state(s._h, ct.byref(out)))
    e2e_s = time.perf_counter() - t1
    name = "PBF" if method == _abi.SPH_PBF else "PCISPH"
    line = {
        "metric": f"{name} steps/s, reference defaults, particle budget {int(args.particles)}",
        "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{name}: pool y<0.1875 + ball r=0.125 in the 10^3 container, "
                               f"timestep {cfg.timestep}, {cfg.substeps} substeps, {cfg.iterations} iterations",
                   "particles": n, "spacing": s.spacing, "kernel_radius": s.kernel_radius, "grid": list(s.grid),
                   "launch": "one CUDA graph per step", "init_s": t_init,
                   "l2": "per-step working set > 126 MB L2 (no flush needed)" if n * 96 > 126e6 else "fits L2"},
        "e2e": {"value": e2e_steps / e2e_s, "unit": "steps/s", "h2d_bytes_per_step": 24 * n,
                "d2h_bytes_per_step": 12 * n, "steps": e2e_steps,
                "path": "aq_sph_upload_state + aq_sph_step + aq_sph_download_state (C ABI), wall clock"},
        "gpu_launches": int(s.launches_per_step() * args.steps),
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = sph_cpu_sample(cfg)
        line["cpu_baseline"] = {"value": cpu["steps"] / cpu["seconds"] * cpu["particles"] / n, "unit": "steps/s",
                                "cores": cpu["threads"], "kind": "port",
                                "sample": f"{cpu['steps']} oracle steps of the same solver at budget 3e5 "
                                          f"({cpu['particles']} particles) in {cpu['seconds']:.1f} s, "
                                          f"scaled by particle count"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    s.close()


def _multiphase_run(args, size: int, dev: int, dist, net=None) -> dict:
    """One timed run of the multiphase workload; with `net` the pressure
    solve starts from the learned warm start (zero-init Jacobi as its
    fallback and judge), else from zero."""
    import torch

    import aquarius_b200 as aq
    from aquarius_b200 import _abi
    vols = [dict(shape="box", min=(0, 0, 0), max=(1, 0.35, 1), phase=0),
            dict(shape="sphere", center=(0.5, 0.75, 0.5), radius=0.12, phase=1)]
    cfg = _abi.make_config((size, size, size), vols, timestep=0.0025, diffusion_coeff=1e-4, phase_count=2,
                           pressure_init=_abi.PRESSURE_LEARNED if net is not None else _abi.PRESSURE_ZERO,
                           solve_mode=_abi.SOLVE_RESIDUAL, rel_residual=1e-4, max_iterations=2000,
                           check_interval=40, device=dev)
    f = aq.Fluid(cfg)
    if net is not None:
        f.set_warm_start(net)
    m0 = f.phase_mass()
    stream = torch.cuda.ExternalStream(f.stream(), device=dev)
    f.step(args.warmup)
    f.synchronize()
    per_step, per_block = f.launch_counts()
    s0 = f.solve_stats()
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.4)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        f.step(args.steps)
        ev1.record(stream)
    ev1.synchronize()
    clk = clocks.stop()
    ms = reduce_max(ev0.elapsed_time(ev1), dist, f"cuda:{dev}")
    s1 = f.solve_stats()
    m1 = f.phase_mass()
    pcg = f.pcg_reference(rel_tol=1e-12, max_iter=400000)
    out = {"ms": ms, "clocks": clk, "particles": f.particleCount,
           "launches": args.steps * per_step + (s1["total_blocks"] - s0["total_blocks"]) * per_block,
           "concentration_mass": {"phase1_initial": m0[1], "phase1_final": m1[1],
                                  "rel_error": abs(m1[1] - m0[1]) / m0[1] if m0[1] else None,
                                  "total_rel_error": abs(sum(m1) - sum(m0)) / sum(m0),
                                  "steps": args.warmup + args.steps},
           "solver": {"sweeps_per_step": (s1["total_sweeps"] - s0["total_sweeps"]) / args.steps,
                      "last_rel_residual": s1["rel_residual"], "converged": s1["converged"],
                      "pressure_rel_error_vs_fp64_pcg": pcg["rel_error"], "pcg_iterations": pcg["iterations"]}}
    if net is not None:
        out["solver"]["warm_start_kept"] = s1["warm_start"] == 1
        out["solver"]["residual_after_20_sweeps"] = {"learned": s1["warm_rel_residual"],
                                                     "zero_init": s1["zero_rel_residual"]}
    f.close()
    return out


def run_multiphase(args, rank: int, world: int, dist):
    """Multiphase FLIP with diffusion at 256^3: a phase-0 pool (concentration
    c = 0) fills y < 0.35, a phase-1 sphere (c = 1) of radius 0.12 sits at
    (0.5, 0.75, 0.5), 8 particles per fluid cell, D = 1e-4, dt = 0.0025,
    Jacobi to relative residual 1e-4 (cap 2000) started from the learned warm
    start (the network fine-tuned on 256^3 pairs, weights/unet_256.bin), 100
    diffusion sweeps; the same run from zero-init pressure is reported beside
    it.  Reports steps/s, the concentration-mass conservation error (the
    change of the phase-1 fraction sum over the run) and the pressure error
    against the FP64 PCG."""
    import torch

    import aquarius_b200 as aq
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    size = args.size if args.size != 128 else 256
    wpath = ROOT / "aquarius_b200" / "weights" / f"unet_{size}.bin"
    plain = _multiphase_run(args, size, dev, dist)
    learned = None
    if wpath.exists() and not args.no_learned:
        net = aq.UNet(device=dev, weights=wpath)
        learned = _multiphase_run(args, size, dev, dist, net)
        learned["weights"] = wpath.name
        learned["time_vs_plain"] = learned["ms"] / plain["ms"]
        net.close()
    main = learned if learned is not None else plain
    init = "learned warm start (weights/" + wpath.name + ")" if learned is not None else "zero-init"
    line = {"metric": "multiphase FLIP steps/s at 256^3 x 8ppc with diffusion, Jacobi to relative residual 1e-4",
            "value": weak_scaling_value(args.steps, world, main["ms"]), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": main["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"multiphase {size}^3 x 8ppc: phase-0 pool y<0.35 + phase-1 sphere r=0.12 at "
                                   f"(0.5,0.75,0.5), D=1e-4, dt=0.0025, 100 diffusion sweeps, {init} Jacobi to "
                                   "rel-res 1e-4 cap 2000",
                       "particles": main["particles"], "l2": "working set > 126 MB L2"},
            "gpu_launches": int(main["launches"]), "clocks": main["clocks"],
            "concentration_mass": main["concentration_mass"], "solver": main["solver"],
            "plain": {"steps_per_s": weak_scaling_value(args.steps, world, plain["ms"]),
                      "ms_per_step": plain["ms"] / args.steps, "solver": plain["solver"],
                      "concentration_mass": plain["concentration_mass"]}}
    if learned is not None:
        line["learned"] = {"weights": learned["weights"], "time_vs_plain": learned["time_vs_plain"]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_profile_case(case: str):
    """Small, fixed cases for single-kernel ncu captures (no JSON line):
    jacobi: the 128^3 workload's system after 3 steps, 6 sweeps of the
    default plan; resident: the same system, 40 sweeps of the resident plan
    (one cooperative launch, 8x40x24 tiles, 384 threads); p2g: the same
    state, the particle-to-grid stage twice; batch-rows: 32 scenes of the batch set, 6 batched sweeps;
    conv: two U-Net inferences at 128^3 on seeded random inputs; mesh: two
    surface meshes of the 128^3 workload's initial particles; pbf / pcisph:
    one step of the solver at particle budget 3e6 (593k particles); render:
    two headless frames (Fluid::draw) of the 128^3 workload's initial
    particles at 1728x864."""
    import numpy as np
    import torch

    import aquarius_b200 as aq
    if case == "jacobi":
        f = aq.Fluid(workload_config(128, "zero"))
        f.step(3)
        f.synchronize()
        print(f.jacobi_plan(), f.benchmark_pressure(6))
        f.close()
    elif case == "p2g":
        from aquarius_b200 import _abi
        f = aq.Fluid(workload_config(128, "zero"))
        f.step(3)
        f.synchronize()
        for _ in range(2):
            f.run_stage(_abi.STAGE_P2G)
        f.synchronize()
        print("p2g ok")
        f.close()
    elif case == "resident":
        f = aq.Fluid(workload_config(128, "zero"))
        f.step(3)
        f.synchronize()
        f.set_jacobi_plan(4, 4, 0)
        print(f.jacobi_plan(), f.benchmark_pressure(40))
        f.close()
    elif case == "batch-rows":
        from aquarius_b200.scenes import batch_configs
        b = aq.Batch(batch_configs(32, seed=BATCH_SEED))
        b.step(2)
        b.synchronize()
        b.set_sweep_plan(8, False)
        print(b.benchmark_pressure(6))
        b.close()
    elif case in ("pbf", "pcisph"):
        from aquarius_b200 import _abi
        m = _abi.SPH_PBF if case == "pbf" else _abi.SPH_PCISPH
        s = aq.Sph(_abi.sph_config(m, max_particle_count=3000000))
        s.step(1)
        s.synchronize()
        print(case, s.n)
        s.close()
    elif case == "mesh":
        f = aq.Fluid(workload_config(128, "zero"))
        f.synchronize()
        for _ in range(2):
            print(len(f.download_mesh(1 << 19)))
        f.close()
    elif case == "render":
        f = aq.Fluid(workload_config(128, "zero"))
        f.synchronize()
        r = aq.Renderer(torch.cuda.current_device())
        r.set_skybox(np.random.default_rng(11).integers(0, 256, (6, 256, 256, 3), dtype=np.uint8))
        dc = aq.draw_command_default(1728, 864, f.getContainerSize(), 128)
        for _ in range(2):
            f.draw(dc, r)
        r.synchronize()
        print("render ok", r.launches())
        r.close()
        f.close()
    elif case == "conv":
        net = aq.UNet(weights=ROOT / "aquarius_b200" / "weights" / "unet_128.bin")
        V = 128 ** 3
        rng = np.random.RandomState(0)
        typ = torch.tensor((rng.rand(V) < 0.5).astype(np.int8), device="cuda")
        rhs = torch.tensor(rng.randn(V).astype(np.float32), device="cuda")
        out = torch.zeros(V, device="cuda")
        torch.cuda.synchronize()
        for _ in range(2):
            net.predict((128, 128, 128), rhs.data_ptr(), typ.data_ptr(), out.data_ptr())
        torch.cuda.synchronize()
        print("conv ok")
        net.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--pressure-init", default="zero", choices=["zero", "carry"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the default Jacobi plan")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start arm")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own kernels (the plain-step comparator)")
    ap.add_argument("--reference-gpu-only", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--profile-case", choices=["jacobi", "resident", "p2g", "batch-rows", "conv", "mesh", "pbf",
                                               "pcisph", "render"],
                    default=None,
                    help="run one small fixed case for an ncu capture and exit")
    ap.add_argument("--workload", default="ball128",
                    choices=["ball128", "ball50", "batch", "multiphase256", "pbf", "pcisph"],
                    help="ball128: the 128^3 scene; ball50: BASELINE config 1 (50^3, 100 sweeps); "
                         "batch: 256 independent scenes of uneven sizes; "
                         "multiphase256: two phases with diffusion at 256^3; pbf / pcisph: the "
                         "particle-only solvers")
    ap.add_argument("--particles", type=float, default=3e7, help="particle budget of the pbf / pcisph workloads")
    ap.add_argument("--scenes", type=int, default=256, help="scenes in the batch workload")
    ap.add_argument("--eager", action="store_true",
                    help="launch the step kernel by kernel instead of one CUDA graph (for launch lists)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.profile_case:
        run_profile_case(args.profile_case)
        return
    if args.reference_gpu_only:
        print(json.dumps(reference_gpu_step_ms(args.size, steps=20 if args.workload == "ball50" else 5,
                                               workload=args.workload)), flush=True)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        if args.workload == "batch":
            run_batch(args, rank, world, dist)
        elif args.workload == "multiphase256":
            run_multiphase(args, rank, world, dist)
        elif args.workload in ("pbf", "pcisph"):
            run_sph(args, rank, world, dist)
        elif args.workload == "ball50":
            run_config1(args, rank, world, dist)
        else:
            run_ours(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
