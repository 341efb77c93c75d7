"""ctypes mirror of include/aquarius_b200.h (structs, enums, state buffers)."""
from __future__ import annotations

import ctypes as ct

import numpy as np

AQ_MAX_VOLUMES = 16
AQ_MAX_PHASES = 4

AQ_OK = 0
AQ_ERR_INVALID_ARGUMENT = 2
AQ_ERR_NOT_CONVERGED = 5
AQ_ERR_NONFINITE = 6
AQ_ERR_TIMEOUT = 8
STATUS_NAMES = {
    0: "AQ_OK",
    1: "AQ_ERR_INVALID_CONFIG",
    2: "AQ_ERR_INVALID_ARGUMENT",
    3: "AQ_ERR_OUT_OF_MEMORY",
    4: "AQ_ERR_CUDA",
    5: "AQ_ERR_NOT_CONVERGED",
    6: "AQ_ERR_NONFINITE",
    7: "AQ_ERR_NO_DEVICE",
    8: "AQ_ERR_TIMEOUT",
}

SHAPE_SPHERE = 0
SHAPE_SQUARE = 1
PRESSURE_CARRY = 0
PRESSURE_ZERO = 1
PRESSURE_LEARNED = 2
SOLVE_FIXED = 0
SOLVE_RESIDUAL = 1

STAGE_G2P_ADVECT = 1
STAGE_SORT = 2
STAGE_P2G = 3
STAGE_DIVERGENCE = 4
STAGE_PRESSURE = 5
STAGE_PROJECT = 6
STAGE_EXTRAPOLATE = 7
STAGE_DIFFUSE = 8
STAGES = {
    "g2p_advect": STAGE_G2P_ADVECT,
    "sort": STAGE_SORT,
    "p2g": STAGE_P2G,
    "divergence": STAGE_DIVERGENCE,
    "pressure": STAGE_PRESSURE,
    "project": STAGE_PROJECT,
    "extrapolate": STAGE_EXTRAPOLATE,
    "diffuse": STAGE_DIFFUSE,
}


class Volume(ct.Structure):
    _fields_ = [
        ("shape", ct.c_int32),
        ("box_min", ct.c_float * 3),
        ("box_max", ct.c_float * 3),
        ("ball_center", ct.c_float * 3),
        ("ball_radius", ct.c_float),
        ("phase", ct.c_int32),
    ]


class Config(ct.Structure):
    _fields_ = [
        ("volume_count", ct.c_int32),
        ("volumes", Volume * AQ_MAX_VOLUMES),
        ("gravity", ct.c_float * 3),
        ("phase_count", ct.c_int32),
        ("phase_densities", ct.c_float * 4),
        ("diffusion_coeff", ct.c_float),
        ("size_x", ct.c_int32),
        ("size_y", ct.c_int32),
        ("size_z", ct.c_int32),
        ("pressure_iterations", ct.c_int32),
        ("diffusion_iterations", ct.c_int32),
        ("timestep", ct.c_float),
        ("flip_coeff", ct.c_float),
        ("particle_jitter", ct.c_float),
        ("domain_size", ct.c_float),
        ("seed", ct.c_uint32),
        ("pressure_init", ct.c_int32),
        ("solve_mode", ct.c_int32),
        ("rel_residual", ct.c_float),
        ("max_iterations", ct.c_int32),
        ("check_interval", ct.c_int32),
        ("device", ct.c_int32),
        ("stream", ct.c_void_p),
    ]


class HostState(ct.Structure):
    _fields_ = [
        ("size_x", ct.c_int32),
        ("size_y", ct.c_int32),
        ("size_z", ct.c_int32),
        ("particle_count", ct.c_int32),
        ("physical_time", ct.c_double),
        ("position", ct.c_void_p),
        ("velocity_p", ct.c_void_p),
        ("fractions", ct.c_void_p),
        ("content", ct.c_void_p),
        ("velocity", ct.c_void_p),
        ("new_velocity", ct.c_void_p),
        ("pressure", ct.c_void_p),
        ("divergence", ct.c_void_p),
        ("particle_count_cell", ct.c_void_p),
        ("has_velocity", ct.c_void_p),
        ("volume_fractions", ct.c_void_p),
        ("new_volume_fractions", ct.c_void_p),
        ("density", ct.c_void_p),
        ("cell_start", ct.c_void_p),
        ("cell_end", ct.c_void_p),
        ("particle_hash", ct.c_void_p),
        ("sort_index", ct.c_void_p),
    ]


class MeshInfo(ct.Structure):
    """aq_mesh_info."""
    _fields_ = [
        ("sdf_size", ct.c_int32 * 3),
        ("mesh_size", ct.c_int32 * 3),
        ("sdf_cell", ct.c_float),
        ("mesh_cell", ct.c_float),
        ("particle_radius", ct.c_float),
    ]


class SolveStats(ct.Structure):
    _fields_ = [
        ("iterations", ct.c_int32),
        ("rel_residual", ct.c_double),
        ("b_norm", ct.c_double),
        ("fluid_cells", ct.c_int32),
        ("converged", ct.c_int32),
        ("blocks", ct.c_int32),
        ("total_sweeps", ct.c_int64),
        ("total_blocks", ct.c_int64),
        ("warm_start", ct.c_int32),
        ("warm_rel_residual", ct.c_double),
        ("zero_rel_residual", ct.c_double),
    ]


class TuneResult(ct.Structure):
    _fields_ = [
        ("levels", ct.c_int32),
        ("rows", ct.c_int32),
        ("x_planes", ct.c_int32),
        ("sweep_us", ct.c_float),
        ("candidates", ct.c_int32),
        ("from_cache", ct.c_int32),
    ]


# name -> (dtype, shape builder(N, C, F))
STATE_FIELDS = {
    "position": (np.float32, lambda n, c, f: (3, n)),
    "velocity_p": (np.float32, lambda n, c, f: (3, n)),
    "fractions": (np.float32, lambda n, c, f: (4, n)),
    "content": (np.int32, lambda n, c, f: (f,)),
    "velocity": (np.float32, lambda n, c, f: (3, f)),
    "new_velocity": (np.float32, lambda n, c, f: (3, f)),
    "pressure": (np.float32, lambda n, c, f: (c,)),
    "divergence": (np.float32, lambda n, c, f: (c,)),
    "particle_count_cell": (np.int32, lambda n, c, f: (c,)),
    "has_velocity": (np.int32, lambda n, c, f: (3, c)),
    "volume_fractions": (np.float32, lambda n, c, f: (4, c)),
    "new_volume_fractions": (np.float32, lambda n, c, f: (4, c)),
    "density": (np.float32, lambda n, c, f: (c,)),
    "cell_start": (np.int32, lambda n, c, f: (c,)),
    "cell_end": (np.int32, lambda n, c, f: (c,)),
    "particle_hash": (np.int32, lambda n, c, f: (n,)),
    "sort_index": (np.int32, lambda n, c, f: (n,)),
}


def grid_counts(sx: int, sy: int, sz: int) -> tuple[int, int]:
    """(cells, nodes) of a sx*sy*sz grid."""
    return sx * sy * sz, (sx + 1) * (sy + 1) * (sz + 1)


def alloc_state(sx: int, sy: int, sz: int, n: int, fields=None) -> dict:
    """Zeroed numpy buffers for the requested fields (all by default)."""
    c, f = grid_counts(sx, sy, sz)
    names = STATE_FIELDS.keys() if fields is None else fields
    out = {}
    for name in names:
        dt, shp = STATE_FIELDS[name]
        out[name] = np.zeros(shp(n, c, f), dtype=dt)
    return out


def make_host_state(sx: int, sy: int, sz: int, n: int, arrays: dict, time: float = 0.0) -> HostState:
    """aq_host_state pointing at the given numpy arrays (others NULL)."""
    st = HostState()
    st.size_x, st.size_y, st.size_z, st.particle_count = sx, sy, sz, n
    st.physical_time = time
    c, f = grid_counts(sx, sy, sz)
    for name, arr in arrays.items():
        dt, shp = STATE_FIELDS[name]
        if arr.dtype != dt or not arr.flags["C_CONTIGUOUS"] or arr.shape != shp(n, c, f):
            raise ValueError(f"state field {name}: need C-contiguous {dt} {shp(n, c, f)}, got {arr.dtype} {arr.shape}")
        setattr(st, name, arr.ctypes.data)
    return st


def default_config_values(cfg: Config) -> Config:
    """Reference defaults (Fluid/FluidConfig.cuh:20-97), filled in Python."""
    ct.memset(ct.byref(cfg), 0, ct.sizeof(cfg))
    cfg.volume_count = 2
    for i, shape in enumerate((SHAPE_SQUARE, SHAPE_SPHERE)):
        v = cfg.volumes[i]
        v.shape = shape
        v.box_min[:] = [0.0, 0.0, 0.0]
        v.box_max[:] = [1.0, 0.1875, 1.0]
        v.ball_center[:] = [0.5, 0.75, 0.5]
        v.ball_radius = 0.125
        v.phase = 0
    cfg.gravity[:] = [0.0, -9.8, 0.0]
    cfg.phase_count = 2
    cfg.phase_densities[:] = [1.0, 1.0, 1.0, 1.0]
    cfg.diffusion_coeff = 0.001
    cfg.size_x = cfg.size_y = cfg.size_z = 50
    cfg.pressure_iterations = 100
    cfg.diffusion_iterations = 100
    cfg.timestep = 0.033
    cfg.flip_coeff = 0.95
    cfg.particle_jitter = 0.05
    cfg.domain_size = 10.0
    cfg.seed = 1
    cfg.pressure_init = PRESSURE_CARRY
    cfg.solve_mode = SOLVE_FIXED
    cfg.rel_residual = 1e-4
    cfg.max_iterations = 2000
    cfg.check_interval = 40
    cfg.device = 0
    cfg.stream = None
    return cfg


def make_config(size=(50, 50, 50), volumes=None, **kw) -> Config:
    """Config with reference defaults, overridden by keyword arguments.

    volumes: list of dicts {shape: 'box'|'sphere', min, max, center, radius, phase}.
    """
    cfg = default_config_values(Config())
    cfg.size_x, cfg.size_y, cfg.size_z = size
    if volumes is not None:
        if len(volumes) > AQ_MAX_VOLUMES:
            raise ValueError("too many volumes")
        cfg.volume_count = len(volumes)
        for i, vd in enumerate(volumes):
            v = cfg.volumes[i]
            v.shape = SHAPE_SPHERE if vd.get("shape") == "sphere" else SHAPE_SQUARE
            v.box_min[:] = list(vd.get("min", (0.0, 0.0, 0.0)))
            v.box_max[:] = list(vd.get("max", (1.0, 0.1875, 1.0)))
            v.ball_center[:] = list(vd.get("center", (0.5, 0.75, 0.5)))
            v.ball_radius = float(vd.get("radius", 0.125))
            v.phase = int(vd.get("phase", 0))
    for k, val in kw.items():
        if k in ("gravity", "phase_densities"):
            getattr(cfg, k)[:] = list(val)
        elif not hasattr(cfg, k):
            raise AttributeError(k)
        else:
            setattr(cfg, k, val)
    return cfg


# ------------------------------------------------------------ SPH solvers
SPH_PBF = 0
SPH_PCISPH = 1


class SphConfig(ct.Structure):
    """aq_sph_config: FluidConfig + ConfigPBF / ConfigPCISPH."""
    _fields_ = [
        ("method", ct.c_int32),
        ("volume_count", ct.c_int32),
        ("volumes", Volume * AQ_MAX_VOLUMES),
        ("gravity", ct.c_float * 3),
        ("timestep", ct.c_float),
        ("substeps", ct.c_int32),
        ("iterations", ct.c_int32),
        ("max_particle_count", ct.c_int32),
        ("particle_jitter", ct.c_float),
        ("stiffness", ct.c_float),
        ("seed", ct.c_uint32),
        ("device", ct.c_int32),
        ("stream", ct.c_void_p),
    ]


class SphState(ct.Structure):
    """aq_sph_state: planar host copies of the particle fields."""
    _fields_ = [
        ("particle_count", ct.c_int32),
        ("physical_time", ct.c_double),
        ("position", ct.c_void_p),
        ("velocity", ct.c_void_p),
        ("density", ct.c_void_p),
        ("rest_density", ct.c_void_p),
        ("last_position", ct.c_void_p),
        ("lambda_", ct.c_void_p),
        ("pressure", ct.c_void_p),
        ("pressure_force", ct.c_void_p),
        ("predicted_position", ct.c_void_p),
        ("predicted_velocity", ct.c_void_p),
    ]


class SphInfo(ct.Structure):
    _fields_ = [
        ("particle_count", ct.c_int32),
        ("particle_spacing", ct.c_float),
        ("kernel_radius", ct.c_float),
        ("grid_size", ct.c_int32 * 3),
        ("container_size", ct.c_float),
    ]


# field name -> components (3: [3][n] plane, 1: [n])
SPH_FIELDS = {
    "position": 3, "velocity": 3, "density": 1, "rest_density": 1, "last_position": 3, "lambda": 1,
    "pressure": 1, "pressure_force": 3, "predicted_position": 3, "predicted_velocity": 3,
}


def sph_config(method=SPH_PBF, volumes=None, **kw) -> SphConfig:
    """aq_sph_config with the reference defaults for the method
    (Fluid/FluidConfig.cuh:52-66, the default volumes and gravity),
    overridden by keyword arguments; volumes as in make_config."""
    c = SphConfig()
    c.method = method
    c.volume_count = 2
    c.volumes[0].shape = SHAPE_SQUARE
    c.volumes[1].shape = SHAPE_SPHERE
    for v in (c.volumes[0], c.volumes[1]):
        v.box_min[:] = [0.0, 0.0, 0.0]
        v.box_max[:] = [1.0, 0.1875, 1.0]
        v.ball_center[:] = [0.5, 0.75, 0.5]
        v.ball_radius = 0.125
    c.gravity[:] = [0.0, -9.8, 0.0]
    if method == SPH_PBF:
        c.timestep, c.substeps, c.iterations = 0.033, 4, 2
    else:
        c.timestep, c.substeps, c.iterations = 0.005, 1, 4
    c.max_particle_count = 300000
    c.particle_jitter = 0.05
    c.stiffness = 15.0
    c.seed = 1
    if volumes is not None:
        c.volume_count = len(volumes)
        for i, vd in enumerate(volumes):
            v = c.volumes[i]
            v.shape = SHAPE_SPHERE if vd.get("shape") == "sphere" else SHAPE_SQUARE
            v.box_min[:] = list(vd.get("min", (0.0, 0.0, 0.0)))
            v.box_max[:] = list(vd.get("max", (1.0, 0.1875, 1.0)))
            v.ball_center[:] = list(vd.get("center", (0.5, 0.75, 0.5)))
            v.ball_radius = float(vd.get("radius", 0.125))
    for k, val in kw.items():
        if k == "gravity":
            c.gravity[:] = list(val)
        elif not hasattr(c, k):
            raise AttributeError(k)
        else:
            setattr(c, k, val)
    return c


def make_sph_state(n: int, arrays: dict, time: float = 0.0) -> SphState:
    st = SphState()
    st.particle_count = n
    st.physical_time = time
    for name, comps in SPH_FIELDS.items():
        a = arrays.get(name)
        if a is not None:
            assert a.dtype == np.float32 and a.size == comps * n and a.flags["C_CONTIGUOUS"], name
            setattr(st, "lambda_" if name == "lambda" else name, a.ctypes.data)
    return st


def alloc_sph_state(n: int, fields=None) -> dict:
    names = SPH_FIELDS.keys() if fields is None else fields
    return {k: np.zeros((SPH_FIELDS[k], n) if SPH_FIELDS[k] == 3 else (n,), np.float32) for k in names}


# ------------------------------------------------------------ headless frame
RENDER_MULTIPHASE_MESH, RENDER_WATER_MESH, RENDER_FLAT_MESH, RENDER_NORMAL_MESH, RENDER_MIRROR_MESH = 0, 1, 2, 3, 4
RENDER_REFRACT_MESH, RENDER_PHASE0_MESH, RENDER_PHASE1_MESH, RENDER_PARTICLES, RENDER_NONE = 5, 6, 7, 8, 9
ENV_SKYBOX, ENV_CORNELL_BOX, ENV_CHESS_BOARD = 0, 1, 2


class DrawCommand(ct.Structure):
    """aq_draw_command: DrawCommand (Rendering/DrawCommand.h:37-59) plus what
    Fluid::draw passes along.  Matrices are column-major (glm layout)."""
    _fields_ = [
        ("view", ct.c_float * 16),
        ("projection", ct.c_float * 16),
        ("camera_position", ct.c_float * 3),
        ("window_width", ct.c_int32),
        ("window_height", ct.c_int32),
        ("fov", ct.c_float),
        ("near_plane", ct.c_float),
        ("far_plane", ct.c_float),
        ("render_mode", ct.c_int32),
        ("environment_mode", ct.c_int32),
        ("light_position", ct.c_float * 3),
        ("container_size", ct.c_float),
        ("cornell_box_size", ct.c_float),
        ("point_radius", ct.c_float),
        ("phase_count", ct.c_int32),
        ("phase_colors", (ct.c_float * 4) * 4),
    ]
