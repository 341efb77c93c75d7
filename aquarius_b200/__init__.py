"""aquarius_b200 — B200-native 3D FLIP step behind the Aquarius solver API.

Python mirror of the reference's plugin surface (AmesingFlank/Aquarius):

    FluidConfig, ConfigFLIP, InitializationVolume, ShapeType
        Fluid/FluidConfig.cuh:16-97
    Fluid.init(config) / simulationStep() / physicalTime / getCenter() /
    getContainerSize() / draw(cmd)
        Fluid/Fluid.h:4-12, Fluid/Fluid_3D.cuh:7-12, Fluid/Fluid_3D_FLIP.cu:316-505

Everything runs in libaquarius_b200.so (hand-written sm_100a kernels behind
the C ABI of include/aquarius_b200.h).  There is no CPU fallback: importing
works without a GPU, but creating a Fluid without the library or a device
raises.
"""
from __future__ import annotations

import ctypes as ct
import dataclasses
import enum
import os
import pathlib
from typing import Optional, Sequence

import numpy as np

from . import _abi

__all__ = [
    "ShapeType", "InitializationVolume", "ConfigFLIP", "FluidConfig", "Fluid", "AquariusError",
    "library_path", "load_library", "STAGES", "Batch", "UNet", "Dataset", "Renderer", "draw_command_default",
]

STAGES = _abi.STAGES
_PKG = pathlib.Path(__file__).resolve().parent
_LIB_NAME = "libaquarius_b200.so"
_lib = None


class AquariusError(RuntimeError):
    """Raised when a C-ABI call returns a status other than AQ_OK."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{_abi.STATUS_NAMES.get(status, status)}: {message}")


def library_path() -> pathlib.Path:
    return _PKG / _LIB_NAME


def load_library() -> ct.CDLL:
    """Loads the in-tree library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = library_path()
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: build it with `python -m aquarius_b200.build`")
    lib = ct.CDLL(str(p))
    P = ct.c_void_p
    sigs = {
        "aq_abi_version": (ct.c_int32, []),
        "aq_last_error": (ct.c_char_p, []),
        "aq_config_default": (ct.c_int, [ct.POINTER(_abi.Config)]),
        "aq_config_validate": (ct.c_int, [ct.POINTER(_abi.Config)]),
        "aq_fluid_create": (ct.c_int, [ct.POINTER(_abi.Config), ct.POINTER(P)]),
        "aq_fluid_step": (ct.c_int, [P, ct.c_int32]),
        "aq_fluid_step_host": (ct.c_int, [P, ct.c_int32, P, P, P, P]),
        "aq_fluid_run_stage": (ct.c_int, [P, ct.c_int32]),
        "aq_fluid_set_graph_mode": (ct.c_int, [P, ct.c_int32]),
        "aq_fluid_synchronize": (ct.c_int, [P]),
        "aq_fluid_time": (ct.c_int, [P, ct.POINTER(ct.c_double)]),
        "aq_fluid_particle_count": (ct.c_int, [P, ct.POINTER(ct.c_int32)]),
        "aq_fluid_container": (ct.c_int, [P, ct.POINTER(ct.c_float), ct.POINTER(ct.c_float)]),
        "aq_fluid_stream": (ct.c_int, [P, ct.POINTER(P)]),
        "aq_fluid_download_state": (ct.c_int, [P, ct.POINTER(_abi.HostState)]),
        "aq_fluid_upload_state": (ct.c_int, [P, ct.POINTER(_abi.HostState)]),
        "aq_fluid_solve_stats": (ct.c_int, [P, ct.POINTER(_abi.SolveStats)]),
        "aq_fluid_test_barrier_timeout": (ct.c_int, [P, ct.c_int32, ct.c_uint32]),
        "aq_selfcheck_division": (ct.c_int, [ct.c_int32, ct.POINTER(ct.c_uint64)]),
        "aq_p2g_set_variant": (ct.c_int, [ct.c_int32]),
        "aq_fluid_pcg_reference": (ct.c_int, [P, ct.c_double, ct.c_int32, P, ct.POINTER(ct.c_double),
                                              ct.POINTER(ct.c_int32), ct.POINTER(ct.c_double)]),
        "aq_fluid_profile_step": (ct.c_int, [P, ct.POINTER(ct.c_float)]),
        "aq_fluid_launches_per_step": (ct.c_int, [P, ct.POINTER(ct.c_int32)]),
        "aq_fluid_launch_counts": (ct.c_int, [P, ct.POINTER(ct.c_int32), ct.POINTER(ct.c_int32)]),
        "aq_fluid_benchmark_pressure": (ct.c_int, [P, ct.c_int32, ct.POINTER(ct.c_float), ct.POINTER(ct.c_int32),
                                                   ct.POINTER(ct.c_int64)]),
        "aq_fluid_set_jacobi_plan": (ct.c_int, [P, ct.c_int32, ct.c_int32, ct.c_int32]),
        "aq_fluid_get_jacobi_plan": (ct.c_int, [P, ct.POINTER(ct.c_int32), ct.POINTER(ct.c_int32),
                                                ct.POINTER(ct.c_int32)]),
        "aq_fluid_autotune": (ct.c_int, [P, ct.c_int32, ct.c_char_p, ct.POINTER(_abi.TuneResult)]),
        "aq_fluid_destroy": (None, [P]),
        "aq_batch_create": (ct.c_int, [ct.POINTER(_abi.Config), ct.c_int32, ct.POINTER(P)]),
        "aq_batch_step": (ct.c_int, [P, ct.c_int32]),
        "aq_batch_synchronize": (ct.c_int, [P]),
        "aq_batch_step_host": (ct.c_int, [P, ct.c_int32, P, P, P, P]),
        "aq_batch_stream": (ct.c_int, [P, ct.POINTER(P)]),
        "aq_batch_scene_count": (ct.c_int32, [P]),
        "aq_batch_scene_info": (ct.c_int, [P, ct.c_int32, ct.POINTER(ct.c_int32), ct.POINTER(ct.c_int64)]),
        "aq_batch_totals": (ct.c_int, [P, ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int64), ct.POINTER(ct.c_int64)]),
        "aq_batch_download_scene": (ct.c_int, [P, ct.c_int32, ct.POINTER(_abi.HostState)]),
        "aq_batch_solve_stats": (ct.c_int, [P, ct.c_int32, ct.POINTER(_abi.SolveStats)]),
        "aq_batch_launch_counts": (ct.c_int, [P, ct.POINTER(ct.c_int32), ct.POINTER(ct.c_int32)]),
        "aq_batch_set_grid_multiple": (ct.c_int, [P, ct.c_int32]),
        "aq_batch_set_sweep_plan": (ct.c_int, [P, ct.c_int32, ct.c_int32]),
        "aq_batch_get_sweep_plan": (ct.c_int, [P, ct.POINTER(ct.c_int32), ct.POINTER(ct.c_int32)]),
        "aq_batch_autotune": (ct.c_int, [P, ct.c_int32, ct.POINTER(ct.c_int32), ct.POINTER(ct.c_int32),
                                         ct.POINTER(ct.c_float)]),
        "aq_batch_benchmark_pressure": (ct.c_int, [P, ct.c_int32, ct.POINTER(ct.c_float), ct.POINTER(ct.c_int64)]),
        "aq_batch_destroy": (None, [P]),
        "aq_unet_create": (ct.c_int, [ct.c_int32, ct.c_uint32, ct.POINTER(P)]),
        "aq_unet_destroy": (None, [P]),
        "aq_unet_parameter_count": (ct.c_int, [P, ct.POINTER(ct.c_int64)]),
        "aq_unet_save": (ct.c_int, [P, ct.c_char_p]),
        "aq_unet_load": (ct.c_int, [P, ct.c_char_p]),
        "aq_unet_get_output_scale": (ct.c_int, [P, ct.POINTER(ct.c_float)]),
        "aq_unet_predict": (ct.c_int, [P, ct.c_int32, ct.c_int32, ct.c_int32, P, P, P, P]),
        "aq_unet_train": (ct.c_int, [P, P, ct.c_int32, ct.c_int32, ct.c_int32, ct.c_float, ct.c_uint32, ct.c_float,
                                     ct.c_float, ct.c_int32, ct.POINTER(ct.c_float)]),
        "aq_unet_evaluate": (ct.c_int, [P, P, ct.c_int32, ct.c_int32, ct.POINTER(ct.c_double)]),
        "aq_unet_gradients": (ct.c_int, [P, P, ct.c_int64]),
        "aq_unet_set_output_scale": (ct.c_int, [P, ct.c_float]),
        "aq_unet_evaluate_warm": (ct.c_int, [P, P, ct.c_int32, ct.c_int32, ct.c_int32, ct.POINTER(ct.c_double)]),
        "aq_fluid_set_warm_start": (ct.c_int, [P, P]),
        "aq_fluid_phase_mass": (ct.c_int, [P, ct.POINTER(ct.c_double)]),
        "aq_fluid_enable_ink": (ct.c_int, [P, ct.POINTER(ct.c_int32)]),
        "aq_fluid_ink_count": (ct.c_int, [P, ct.POINTER(ct.c_int32)]),
        "aq_fluid_download_ink": (ct.c_int, [P, P, P]),
        "aq_fluid_upload_ink": (ct.c_int, [P, P, P]),
        "aq_fluid_ink_advance": (ct.c_int, [P]),
        "aq_sph_config_default": (ct.c_int, [ct.c_int32, P]),
        "aq_sph_create": (ct.c_int, [P, ct.POINTER(P)]),
        "aq_sph_destroy": (None, [P]),
        "aq_sph_info_get": (ct.c_int, [P, P]),
        "aq_sph_step": (ct.c_int, [P, ct.c_int32]),
        "aq_sph_synchronize": (ct.c_int, [P]),
        "aq_sph_launches_per_step": (ct.c_int, [P, ct.POINTER(ct.c_int32)]),
        "aq_sph_download_state": (ct.c_int, [P, P]),
        "aq_sph_upload_state": (ct.c_int, [P, P]),
        "aq_fluid_mesh_info": (ct.c_int, [P, P]),
        "aq_fluid_mesh": (ct.c_int, [P, P, ct.c_int64, ct.POINTER(ct.c_int32)]),
        "aq_fluid_download_mesh": (ct.c_int, [P, P, ct.c_int64, ct.POINTER(ct.c_int32)]),
        "aq_fluid_download_sdf": (ct.c_int, [P, P]),
        "aq_dataset_create": (ct.c_int, [ct.c_int32, ct.c_int32, ct.c_int32, ct.c_int32, ct.c_int32, ct.POINTER(P)]),
        "aq_dataset_destroy": (None, [P]),
        "aq_dataset_count": (ct.c_int32, [P]),
        "aq_dataset_add_fluid": (ct.c_int, [P, P, ct.c_double, ct.c_int32, ct.POINTER(ct.c_int32)]),
        "aq_dataset_target_rms": (ct.c_int, [P, ct.c_int32, ct.c_int32, ct.POINTER(ct.c_double)]),
        "aq_dataset_get": (ct.c_int, [P, ct.c_int32, P, P, P]),
        "aq_draw_command_default": (ct.c_int, [P, ct.c_int32, ct.c_int32, ct.c_float, ct.c_int32]),
        "aq_fluid_points_vbo": (ct.c_int, [P, P]),
        "aq_renderer_create": (ct.c_int, [ct.c_int32, P, ct.POINTER(P)]),
        "aq_renderer_destroy": (None, [P]),
        "aq_renderer_set_skybox": (ct.c_int, [P, P, ct.c_int32]),
        "aq_renderer_set_logo": (ct.c_int, [P, P, ct.c_int32, ct.c_int32]),
        "aq_renderer_draw": (ct.c_int, [P, P, P, ct.c_int32, P, ct.c_int64, P]),
        "aq_renderer_synchronize": (ct.c_int, [P]),
        "aq_renderer_download_phase_thickness": (ct.c_int, [P, P]),
        "aq_renderer_download_image": (ct.c_int, [P, P]),
        "aq_renderer_launches": (ct.c_int, [P, ct.POINTER(ct.c_int32)]),
        "aq_fluid_draw": (ct.c_int, [P, P, P, P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(status: int):
    if status != _abi.AQ_OK:
        msg = load_library().aq_last_error()
        raise AquariusError(status, msg.decode() if msg else "")


class ShapeType(enum.IntEnum):
    """ShapeType {Sphere, Square} (Fluid/FluidConfig.cuh:16-18)."""
    Sphere = _abi.SHAPE_SPHERE
    Square = _abi.SHAPE_SQUARE


@dataclasses.dataclass
class InitializationVolume:
    """InitializationVolume (Fluid/FluidConfig.cuh:20-38); [0,1] coordinates."""
    shapeType: ShapeType = ShapeType.Square
    boxMin: Sequence[float] = (0.0, 0.0, 0.0)
    boxMax: Sequence[float] = (1.0, 0.1875, 1.0)
    ballCenter: Sequence[float] = (0.5, 0.75, 0.5)
    ballRadius: float = 0.125
    phase: int = 0


@dataclasses.dataclass
class ConfigFLIP:
    """ConfigFLIP (Fluid/FluidConfig.cuh:41-50)."""
    sizeX: int = 50
    sizeY: int = 50
    sizeZ: int = 50
    pressureIterations: int = 100
    diffusionIterations: int = 100
    timestep: float = 0.033
    FLIPcoeff: float = 0.95
    particleJitter: float = 0.05


def _default_volumes():
    return [InitializationVolume(ShapeType.Square), InitializationVolume(ShapeType.Sphere)]


@dataclasses.dataclass
class FluidConfig:
    """FluidConfig (Fluid/FluidConfig.cuh:68-97) plus this library's solver options.

    Extensions (no reference counterpart): gridPhysicalSize (the reference's
    Fluid member, 10), seed (rand() seed; the reference's unseeded rand() is
    seed 1), pressureInit ('carry' = reference, 'zero'), solveMode ('fixed' =
    reference, 'residual'), relResidual, maxIterations, checkInterval,
    device, stream (a cudaStream_t as int, or None).
    """
    method: str = "FLIP"
    initialVolumes: list = dataclasses.field(default_factory=_default_volumes)
    gravity: Sequence[float] = (0.0, -9.8, 0.0)
    phaseCount: int = 2
    phaseDensities: Sequence[float] = (1.0, 1.0, 1.0, 1.0)
    diffusionCoeff: float = 0.001
    FLIP: ConfigFLIP = dataclasses.field(default_factory=ConfigFLIP)
    gridPhysicalSize: float = 10.0
    seed: int = 1
    pressureInit: str = "carry"
    solveMode: str = "fixed"
    relResidual: float = 1e-4
    maxIterations: int = 2000
    checkInterval: int = 40
    device: int = 0
    stream: Optional[int] = None

    def to_c(self) -> _abi.Config:
        if self.method != "FLIP":
            raise ValueError(f"method {self.method!r}: this library implements the FLIP solver only")
        vols = []
        for v in self.initialVolumes:
            vols.append(dict(shape="sphere" if ShapeType(v.shapeType) == ShapeType.Sphere else "box",
                             min=tuple(v.boxMin), max=tuple(v.boxMax), center=tuple(v.ballCenter),
                             radius=v.ballRadius, phase=v.phase))
        f = self.FLIP
        return _abi.make_config(
            (f.sizeX, f.sizeY, f.sizeZ), vols, gravity=tuple(self.gravity), phase_count=self.phaseCount,
            phase_densities=tuple(self.phaseDensities), diffusion_coeff=self.diffusionCoeff,
            pressure_iterations=f.pressureIterations, diffusion_iterations=f.diffusionIterations,
            timestep=f.timestep, flip_coeff=f.FLIPcoeff, particle_jitter=f.particleJitter,
            domain_size=self.gridPhysicalSize, seed=self.seed,
            pressure_init={"carry": _abi.PRESSURE_CARRY, "zero": _abi.PRESSURE_ZERO,
                           "learned": _abi.PRESSURE_LEARNED}[self.pressureInit],
            solve_mode={"fixed": _abi.SOLVE_FIXED, "residual": _abi.SOLVE_RESIDUAL}[self.solveMode],
            rel_residual=self.relResidual, max_iterations=self.maxIterations,
            check_interval=self.checkInterval, device=self.device, stream=self.stream)


class Fluid:
    """Fluid_3D_FLIP::Fluid: init(config) then simulationStep() per frame."""

    def __init__(self, config: Optional[FluidConfig] = None):
        self._lib = load_library()
        self._h = ct.c_void_p()
        self.config: Optional[FluidConfig] = None
        self._cfg_c: Optional[_abi.Config] = None
        if config is not None:
            self.init(config)

    # -- reference surface ---------------------------------------------------
    def init(self, config: FluidConfig):
        """Fluid::init (Fluid/Fluid_3D_FLIP.cu:435-505)."""
        self.close()
        cfg_c = config.to_c() if isinstance(config, FluidConfig) else config
        _check(self._lib.aq_fluid_create(ct.byref(cfg_c), ct.byref(self._h)))
        self.config = config if isinstance(config, FluidConfig) else None
        self._cfg_c = cfg_c
        n = ct.c_int32()
        _check(self._lib.aq_fluid_particle_count(self._h, ct.byref(n)))
        self.particleCount = n.value
        self.size = (cfg_c.size_x, cfg_c.size_y, cfg_c.size_z)

    def simulationStep(self):
        """Fluid::simulationStep (Fluid/Fluid_3D_FLIP.cu:316-352), asynchronous."""
        _check(self._lib.aq_fluid_step(self._h, 1))

    @property
    def physicalTime(self) -> float:
        t = ct.c_double()
        _check(self._lib.aq_fluid_time(self._h, ct.byref(t)))
        return t.value

    def getCenter(self):
        c = (ct.c_float * 3)()
        _check(self._lib.aq_fluid_container(self._h, c, None))
        return tuple(c)

    def getContainerSize(self) -> float:
        s = ct.c_float()
        _check(self._lib.aq_fluid_container(self._h, None, ct.byref(s)))
        return s.value

    # -- extensions -----------------------------------------------------------
    def step(self, n: int = 1):
        _check(self._lib.aq_fluid_step(self._h, n))

    def step_host(self, n: int, position_in=None, velocity_in=None, position_out=None, velocity_out=None):
        """Steps with particle state in host arrays ([3][N] float32)."""
        def ptr(a):
            return None if a is None else a.ctypes.data
        _check(self._lib.aq_fluid_step_host(self._h, n, ptr(position_in), ptr(velocity_in), ptr(position_out),
                                            ptr(velocity_out)))

    def set_graph_mode(self, use_graph: bool):
        """True (default): one CUDA-graph launch per step; False: kernel by kernel."""
        _check(self._lib.aq_fluid_set_graph_mode(self._h, 1 if use_graph else 0))

    def run_stage(self, stage):
        k = STAGES[stage] if isinstance(stage, str) else int(stage)
        _check(self._lib.aq_fluid_run_stage(self._h, k))

    def synchronize(self):
        _check(self._lib.aq_fluid_synchronize(self._h))

    def stream(self) -> int:
        s = ct.c_void_p()
        _check(self._lib.aq_fluid_stream(self._h, ct.byref(s)))
        return s.value or 0

    def download_state(self, fields=None) -> dict:
        sx, sy, sz = self.size
        arrs = _abi.alloc_state(sx, sy, sz, self.particleCount, fields)
        st = _abi.make_host_state(sx, sy, sz, self.particleCount, arrs)
        _check(self._lib.aq_fluid_download_state(self._h, ct.byref(st)))
        arrs["physical_time"] = st.physical_time
        return arrs

    def upload_state(self, state: dict):
        sx, sy, sz = self.size
        arrs = {k: np.ascontiguousarray(v) for k, v in state.items() if k in _abi.STATE_FIELDS}
        st = _abi.make_host_state(sx, sy, sz, self.particleCount, arrs, float(state.get("physical_time", 0.0)))
        _check(self._lib.aq_fluid_upload_state(self._h, ct.byref(st)))

    def solve_stats(self) -> dict:
        """Statistics of the last pressure solve.  "status" is the call's
        aq_status name: AQ_ERR_NOT_CONVERGED (residual mode stopped at its cap)
        and AQ_ERR_NONFINITE are reported there, other errors raise."""
        s = _abi.SolveStats()
        rc = self._lib.aq_fluid_solve_stats(self._h, ct.byref(s))
        if rc not in (_abi.AQ_OK, _abi.AQ_ERR_NOT_CONVERGED, _abi.AQ_ERR_NONFINITE):
            _check(rc)
        d = _solve_stats_dict(s)
        d["status"] = _abi.STATUS_NAMES.get(rc, str(rc))
        return d

    def test_barrier_timeout(self, withhold_cta: int = -1, spin_limit: int = 0):
        """Test hook of the bounded grid-barrier waits of the persistent
        solves (aq_fluid_test_barrier_timeout); (-1, 0) switches it off."""
        _check(self._lib.aq_fluid_test_barrier_timeout(self._h, withhold_cta, spin_limit))

    def phase_mass(self) -> list:
        """Sum over particles of the volume fractions of each of the 4 phases."""
        m = (ct.c_double * 4)()
        _check(self._lib.aq_fluid_phase_mass(self._h, m))
        return list(m)

    def enable_ink(self) -> int:
        """Seeds the ink particles (Fluid::initInkRenderer) once; every later
        step then ends by advancing them.  Returns the ink count."""
        n = ct.c_int32()
        _check(self._lib.aq_fluid_enable_ink(self._h, ct.byref(n)))
        return n.value

    @property
    def ink_count(self) -> int:
        n = ct.c_int32()
        _check(self._lib.aq_fluid_ink_count(self._h, ct.byref(n)))
        return n.value

    def get_ink(self) -> dict:
        """Ink positions and velocities as [3, n] float32 arrays."""
        n = self.ink_count
        pos = np.zeros((3, n), np.float32)
        vel = np.zeros((3, n), np.float32)
        _check(self._lib.aq_fluid_download_ink(self._h, pos.ctypes.data, vel.ctypes.data))
        return {"position": pos, "velocity": vel}

    def set_ink(self, position=None, velocity=None):
        n = self.ink_count
        p = None if position is None else np.ascontiguousarray(position, np.float32).reshape(3, n)
        v = None if velocity is None else np.ascontiguousarray(velocity, np.float32).reshape(3, n)
        _check(self._lib.aq_fluid_upload_ink(self._h, None if p is None else p.ctypes.data,
                                              None if v is None else v.ctypes.data))

    def ink_advance(self):
        """transferToInkParticles + moveInkParticles on the current grids."""
        _check(self._lib.aq_fluid_ink_advance(self._h))

    def mesh_info(self) -> dict:
        """Grid sizes of the surface mesher (Mesher as Fluid::init builds it)."""
        info = _abi.MeshInfo()
        _check(self._lib.aq_fluid_mesh_info(self._h, ct.byref(info)))
        return {"sdf": tuple(info.sdf_size), "mesh": tuple(info.mesh_size), "h_sdf": info.sdf_cell,
                "h_mesh": info.mesh_cell, "radius": info.particle_radius}

    def download_mesh(self, capacity=None) -> np.ndarray:
        """Meshes the current particles; the occupied-cube records, [k, 15, 6]
        (position xyz, normal xyz per vertex slot; unused slots zero)."""
        n = ct.c_int32()
        if capacity is None:
            _check(self._lib.aq_fluid_download_mesh(self._h, None, 0, ct.byref(n)))
            capacity = n.value
        out = np.zeros((max(int(capacity), 1), 15, 6), np.float32)
        _check(self._lib.aq_fluid_download_mesh(self._h, out.ctypes.data, int(capacity), ct.byref(n)))
        return out[: min(n.value, int(capacity))]

    def mesh_into(self, device_ptr: int, capacity_records: int) -> int:
        """Meshes into a device buffer of capacity_records records (the
        reference's mesh VBO layout); returns the occupied-cube count."""
        n = ct.c_int32()
        _check(self._lib.aq_fluid_mesh(self._h, ct.c_void_p(device_ptr), int(capacity_records), ct.byref(n)))
        return n.value

    def points_vbo_into(self, device_ptr: int):
        """updatePositionsAndPhasesVBO: 7 floats per particle into a device buffer."""
        _check(self._lib.aq_fluid_points_vbo(self._h, ct.c_void_p(device_ptr)))

    def draw(self, drawCommand: Optional[_abi.DrawCommand] = None, renderer: Optional["Renderer"] = None,
             device_ptr: Optional[int] = None):
        """Fluid::draw(drawCommand) (Fluid/Fluid_3D_FLIP.cu:396-430), headless:
        mesh (mesh modes), point VBO and one frame, into device_ptr (W*H*4
        bytes) or, when None, the renderer's own image (renderer.image()
        downloads it).  Without a renderer the fluid's own is used (made on
        first use); without a draw command nothing is drawn.  Returns the
        renderer."""
        if drawCommand is None:
            return renderer
        if renderer is None:
            if getattr(self, "_renderer", None) is None:
                self._renderer = Renderer(int(self._cfg_c.device))
            renderer = self._renderer
        _check(self._lib.aq_fluid_draw(self._h, renderer._h, ct.byref(drawCommand),
                                       None if device_ptr is None else ct.c_void_p(device_ptr)))
        renderer._last = (drawCommand.window_height, drawCommand.window_width)
        return renderer

    def download_sdf(self) -> np.ndarray:
        """The last mesh's SDF grid, [sdf_x, sdf_y, sdf_z]."""
        info = self.mesh_info()
        out = np.zeros(info["sdf"], np.float32)
        _check(self._lib.aq_fluid_download_sdf(self._h, out.ctypes.data))
        return out

    def set_warm_start(self, net):
        """Attaches the network AQ_PRESSURE_LEARNED ('learned') uses (None detaches)."""
        self._net = net
        _check(self._lib.aq_fluid_set_warm_start(self._h, None if net is None else net.handle))

    def pcg_reference(self, rel_tol: float = 1e-12, max_iter: int = 100000, want_pressure: bool = False):
        """FP64 PCG solve of the current pressure system; returns the relative
        L2 error of the fluid's pressure against it over fluid cells."""
        out = np.zeros(self.size[0] * self.size[1] * self.size[2], np.float32) if want_pressure else None
        err, res = ct.c_double(), ct.c_double()
        it = ct.c_int32()
        _check(self._lib.aq_fluid_pcg_reference(self._h, rel_tol, max_iter, None if out is None else out.ctypes.data,
                                                ct.byref(err), ct.byref(it), ct.byref(res)))
        d = {"rel_error": err.value, "iterations": it.value, "residual": res.value}
        if out is not None:
            d["pressure"] = out
        return d

    def profile_step(self) -> dict:
        ms = (ct.c_float * 8)()
        _check(self._lib.aq_fluid_profile_step(self._h, ms))
        return {name: ms[k - 1] for name, k in STAGES.items()}

    def launches_per_step(self) -> int:
        n = ct.c_int32()
        _check(self._lib.aq_fluid_launches_per_step(self._h, ct.byref(n)))
        return n.value

    def set_jacobi_plan(self, levels: int, rows: int, x_planes: int):
        _check(self._lib.aq_fluid_set_jacobi_plan(self._h, levels, rows, x_planes))

    def jacobi_plan(self) -> tuple:
        a, b, c = ct.c_int32(), ct.c_int32(), ct.c_int32()
        _check(self._lib.aq_fluid_get_jacobi_plan(self._h, ct.byref(a), ct.byref(b), ct.byref(c)))
        return a.value, b.value, c.value

    def autotune(self, sweeps_per_trial: int = 200, cache_path=None) -> dict:
        """Times the candidate Jacobi plans on the current system and keeps the
        fastest (optionally cached per GPU and grid in a JSON file)."""
        r = _abi.TuneResult()
        path = None if cache_path is None else str(cache_path).encode()
        _check(self._lib.aq_fluid_autotune(self._h, sweeps_per_trial, path, ct.byref(r)))
        return {"plan": (r.levels, r.rows, r.x_planes), "sweep_us": r.sweep_us, "candidates": r.candidates,
                "from_cache": bool(r.from_cache)}

    def launch_counts(self) -> tuple:
        a, b = ct.c_int32(), ct.c_int32()
        _check(self._lib.aq_fluid_launch_counts(self._h, ct.byref(a), ct.byref(b)))
        return a.value, b.value

    def benchmark_pressure(self, sweeps: int) -> dict:
        """Times `sweeps` Jacobi sweeps of the current system (CUDA events)."""
        ms, nl, cells = ct.c_float(), ct.c_int32(), ct.c_int64()
        _check(self._lib.aq_fluid_benchmark_pressure(self._h, sweeps, ct.byref(ms), ct.byref(nl), ct.byref(cells)))
        return {"ms": ms.value, "launches": nl.value, "cells_per_sweep": cells.value}

    def close(self):
        r = getattr(self, "_renderer", None)
        if r is not None:
            r.close()
            self._renderer = None
        if getattr(self, "_h", None) and self._h.value:
            self._lib.aq_fluid_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _solve_stats_dict(s) -> dict:
    return {"iterations": s.iterations, "rel_residual": s.rel_residual, "b_norm": s.b_norm,
            "fluid_cells": s.fluid_cells, "converged": bool(s.converged), "blocks": s.blocks,
            "total_sweeps": s.total_sweeps, "total_blocks": s.total_blocks, "warm_start": s.warm_start,
            "warm_rel_residual": s.warm_rel_residual, "zero_rel_residual": s.zero_rel_residual}


class Sph:
    """Fluid_3D_PBF::Fluid / Fluid_3D_PCISPH::Fluid: init(config) then
    simulationStep() per frame (aq_sph_* in include/aquarius_b200.h)."""

    PBF = _abi.SPH_PBF
    PCISPH = _abi.SPH_PCISPH

    def __init__(self, config: _abi.SphConfig):
        self._lib = load_library()
        self._h = ct.c_void_p()
        self._cfg = config
        _check(self._lib.aq_sph_create(ct.byref(config), ct.byref(self._h)))
        info = _abi.SphInfo()
        _check(self._lib.aq_sph_info_get(self._h, ct.byref(info)))
        self.n = info.particle_count
        self.particleCount = info.particle_count
        self.spacing = info.particle_spacing
        self.kernel_radius = info.kernel_radius
        self.grid = tuple(info.grid_size)

    @staticmethod
    def default_config(method: int) -> _abi.SphConfig:
        c = _abi.SphConfig()
        _check(load_library().aq_sph_config_default(method, ct.byref(c)))
        return c

    def simulationStep(self):
        _check(self._lib.aq_sph_step(self._h, 1))

    def step(self, n: int = 1):
        _check(self._lib.aq_sph_step(self._h, int(n)))

    def synchronize(self):
        _check(self._lib.aq_sph_synchronize(self._h))

    def launches_per_step(self) -> int:
        v = ct.c_int32()
        _check(self._lib.aq_sph_launches_per_step(self._h, ct.byref(v)))
        return v.value

    def get_state(self, fields=None) -> dict:
        arrs = _abi.alloc_sph_state(self.n, fields)
        st = _abi.make_sph_state(self.n, arrs)
        _check(self._lib.aq_sph_download_state(self._h, ct.byref(st)))
        arrs["physical_time"] = st.physical_time
        return arrs

    def set_state(self, state: dict):
        arrs = {k: np.ascontiguousarray(v, np.float32) for k, v in state.items() if k in _abi.SPH_FIELDS}
        st = _abi.make_sph_state(self.n, arrs, float(state.get("physical_time", 0.0)))
        _check(self._lib.aq_sph_upload_state(self._h, ct.byref(st)))

    def close(self):
        if self._h:
            self._lib.aq_sph_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def draw_command_default(width: int, height: int, domain_size: float, size_y: int) -> _abi.DrawCommand:
    """main.cu's first-frame DrawCommand for a fluid of physical size
    domain_size with size_y cells along y (aq_draw_command_default)."""
    dc = _abi.DrawCommand()
    _check(load_library().aq_draw_command_default(ct.byref(dc), int(width), int(height), float(domain_size),
                                                  int(size_y)))
    return dc


class Renderer:
    """The headless frame of the reference's renderer (aq_renderer_* in
    include/aquarius_b200.h): Skybox, Container, PointSprites and
    FluidMeshRenderer draws as CUDA kernels writing an RGBA8 image, row 0 at
    the bottom."""

    def __init__(self, device: int = 0):
        self._lib = load_library()
        self._h = ct.c_void_p()
        _check(self._lib.aq_renderer_create(int(device), None, ct.byref(self._h)))
        self._last = None

    def set_skybox(self, faces: Optional[np.ndarray]):
        """faces: uint8 [6, F, F, 3] in the order posx, negx, posy, negy, posz, negz."""
        if faces is None:
            _check(self._lib.aq_renderer_set_skybox(self._h, None, 0))
            return
        f = np.ascontiguousarray(faces, np.uint8)
        assert f.ndim == 4 and f.shape[0] == 6 and f.shape[1] == f.shape[2] and f.shape[3] == 3
        _check(self._lib.aq_renderer_set_skybox(self._h, f.ctypes.data, f.shape[1]))

    def set_logo(self, img: Optional[np.ndarray]):
        """img: uint8 [H, W, 3], first row at t = 0."""
        if img is None:
            _check(self._lib.aq_renderer_set_logo(self._h, None, 0, 0))
            return
        a = np.ascontiguousarray(img, np.uint8)
        _check(self._lib.aq_renderer_set_logo(self._h, a.ctypes.data, a.shape[1], a.shape[0]))

    def draw(self, command: _abi.DrawCommand, points_ptr: int = 0, n_points: int = 0, mesh_ptr: int = 0,
             n_vertices: int = 0, rgba_ptr: Optional[int] = None):
        """One frame from device VBOs into a device image (or the renderer's own)."""
        _check(self._lib.aq_renderer_draw(self._h, ct.byref(command), ct.c_void_p(points_ptr) if points_ptr else None,
                                          int(n_points), ct.c_void_p(mesh_ptr) if mesh_ptr else None,
                                          int(n_vertices), None if rgba_ptr is None else ct.c_void_p(rgba_ptr)))
        self._last = (command.window_height, command.window_width)

    def synchronize(self):
        _check(self._lib.aq_renderer_synchronize(self._h))

    def image(self) -> np.ndarray:
        """The last frame, uint8 [H, W, 4], row 0 at the bottom."""
        h, w = self._last
        out = np.empty((h, w, 4), np.uint8)
        _check(self._lib.aq_renderer_download_image(self._h, out.ctypes.data))
        return out

    def phase_thickness(self) -> np.ndarray:
        """The last frame's phase-thickness texture, float32 [H, W, 4]."""
        h, w = self._last
        out = np.empty((h, w, 4), np.float32)
        _check(self._lib.aq_renderer_download_phase_thickness(self._h, out.ctypes.data))
        return out

    def launches(self) -> int:
        v = ct.c_int32()
        _check(self._lib.aq_renderer_launches(self._h, ct.byref(v)))
        return v.value

    def close(self):
        if self._h:
            self._lib.aq_renderer_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many independent single-phase scenes stepped together (no reference
    counterpart): one launch per stage over all scenes, one CUDA graph per
    step.  Scene s evolves bit for bit as Fluid(configs[s]) with the default
    Jacobi plan."""

    def __init__(self, configs):
        self._lib = load_library()
        self._h = ct.c_void_p()
        cs = [c.to_c() if isinstance(c, FluidConfig) else c for c in configs]
        arr = (_abi.Config * len(cs))(*cs)
        _check(self._lib.aq_batch_create(arr, len(cs), ct.byref(self._h)))
        self.scene_count = self._lib.aq_batch_scene_count(self._h)
        self.sizes, self.particle_counts = [], []
        for i in range(self.scene_count):
            sz = (ct.c_int32 * 3)()
            n = ct.c_int64()
            _check(self._lib.aq_batch_scene_info(self._h, i, sz, ct.byref(n)))
            self.sizes.append(tuple(sz))
            self.particle_counts.append(n.value)

    def step(self, n: int = 1):
        _check(self._lib.aq_batch_step(self._h, n))

    def synchronize(self):
        _check(self._lib.aq_batch_synchronize(self._h))

    def step_host(self, n: int, position_in=None, velocity_in=None, position_out=None, velocity_out=None):
        """Steps with the particle state of all scenes in host arrays ([3][N],
        scenes concatenated in batch order); synchronous."""
        def ptr(a):
            return None if a is None else a.ctypes.data
        _check(self._lib.aq_batch_step_host(self._h, n, ptr(position_in), ptr(velocity_in), ptr(position_out),
                                            ptr(velocity_out)))

    def stream(self) -> int:
        s = ct.c_void_p()
        _check(self._lib.aq_batch_stream(self._h, ct.byref(s)))
        return s.value or 0

    def totals(self) -> dict:
        c, f, p = ct.c_int64(), ct.c_int64(), ct.c_int64()
        _check(self._lib.aq_batch_totals(self._h, ct.byref(c), ct.byref(f), ct.byref(p)))
        return {"cells": c.value, "nodes": f.value, "particles": p.value}

    def download_scene(self, scene: int, fields=None) -> dict:
        sx, sy, sz = self.sizes[scene]
        n = self.particle_counts[scene]
        arrs = _abi.alloc_state(sx, sy, sz, n, fields)
        st = _abi.make_host_state(sx, sy, sz, n, arrs)
        _check(self._lib.aq_batch_download_scene(self._h, scene, ct.byref(st)))
        arrs["physical_time"] = st.physical_time
        return arrs

    def solve_stats(self, scene: int) -> dict:
        s = _abi.SolveStats()
        _check(self._lib.aq_batch_solve_stats(self._h, scene, ct.byref(s)))
        return _solve_stats_dict(s)

    def launch_counts(self) -> tuple:
        a, b = ct.c_int32(), ct.c_int32()
        _check(self._lib.aq_batch_launch_counts(self._h, ct.byref(a), ct.byref(b)))
        return a.value, b.value

    def set_grid_multiple(self, multiple: int):
        _check(self._lib.aq_batch_set_grid_multiple(self._h, multiple))

    def set_sweep_plan(self, x_planes: int, pipelined: bool = False):
        _check(self._lib.aq_batch_set_sweep_plan(self._h, x_planes, int(pipelined)))

    def sweep_plan(self) -> tuple:
        a, b = ct.c_int32(), ct.c_int32()
        _check(self._lib.aq_batch_get_sweep_plan(self._h, ct.byref(a), ct.byref(b)))
        return a.value, bool(b.value)

    def autotune(self, sweeps_per_trial: int = 100) -> dict:
        """Times every batched sweep plan on the current systems and keeps the fastest."""
        xp, pp, us = ct.c_int32(), ct.c_int32(), ct.c_float()
        _check(self._lib.aq_batch_autotune(self._h, sweeps_per_trial, ct.byref(xp), ct.byref(pp), ct.byref(us)))
        return {"x_planes": xp.value, "pipelined": bool(pp.value), "sweep_us": us.value}

    def benchmark_pressure(self, sweeps: int) -> dict:
        ms, cells = ct.c_float(), ct.c_int64()
        _check(self._lib.aq_batch_benchmark_pressure(self._h, sweeps, ct.byref(ms), ct.byref(cells)))
        return {"ms": ms.value, "cells_per_sweep": cells.value}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.aq_batch_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class UNet:
    """The learned pressure warm start's network (no reference counterpart):
    a 3-level 3D U-Net in BF16 with FP32 accumulation, trained and run by the
    library's own kernels."""

    def __init__(self, device: int = 0, seed: int = 1, weights=None):
        self._lib = load_library()
        self._h = ct.c_void_p()
        _check(self._lib.aq_unet_create(device, seed, ct.byref(self._h)))
        if weights is not None:
            self.load(weights)

    @property
    def handle(self):
        return self._h

    def parameter_count(self) -> int:
        n = ct.c_int64()
        _check(self._lib.aq_unet_parameter_count(self._h, ct.byref(n)))
        return n.value

    def save(self, path):
        _check(self._lib.aq_unet_save(self._h, str(path).encode()))

    def load(self, path):
        _check(self._lib.aq_unet_load(self._h, str(path).encode()))

    def output_scale(self) -> float:
        v = ct.c_float()
        _check(self._lib.aq_unet_get_output_scale(self._h, ct.byref(v)))
        return v.value

    def predict(self, size, rhs_ptr: int, type_ptr: int, out_ptr: int, stream: int = 0):
        _check(self._lib.aq_unet_predict(self._h, *size, rhs_ptr, type_ptr, out_ptr, stream or None))

    def train(self, ds: "Dataset", first: int, count: int, steps: int, lr: float = 1e-3, seed: int = 1,
              out_scale: float = 0.0, residual_weight: float = 0.0, residual_sweeps: int = 20) -> float:
        loss = ct.c_float()
        _check(self._lib.aq_unet_train(self._h, ds._h, first, count, steps, lr, seed, out_scale, residual_weight,
                                       residual_sweeps, ct.byref(loss)))
        return loss.value

    def evaluate(self, ds: "Dataset", first: int, count: int) -> float:
        e = ct.c_double()
        _check(self._lib.aq_unet_evaluate(self._h, ds._h, first, count, ct.byref(e)))
        return e.value

    def set_output_scale(self, scale: float):
        _check(self._lib.aq_unet_set_output_scale(self._h, scale))

    def evaluate_warm(self, ds: "Dataset", first: int, count: int, sweeps: int = 20) -> float:
        """Mean (residual after `sweeps` sweeps from the prediction) / (from zero)."""
        r = ct.c_double()
        _check(self._lib.aq_unet_evaluate_warm(self._h, ds._h, first, count, sweeps, ct.byref(r)))
        return r.value

    def gradients(self) -> np.ndarray:
        out = np.zeros(self.parameter_count(), np.float32)
        _check(self._lib.aq_unet_gradients(self._h, out.ctypes.data, out.size))
        return out

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.aq_unet_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Dataset:
    """Device-resident (rhs, fluid mark) -> FP64-PCG pressure pairs of one grid size."""

    def __init__(self, size, capacity: int, device: int = 0):
        self._lib = load_library()
        self._h = ct.c_void_p()
        self.size = tuple(size)
        _check(self._lib.aq_dataset_create(*self.size, capacity, device, ct.byref(self._h)))

    def __len__(self):
        return self._lib.aq_dataset_count(self._h)

    def add_fluid(self, fluid: Fluid, pcg_rel_tol: float = 1e-10, pcg_max_iter: int = 100000) -> int:
        it = ct.c_int32()
        _check(self._lib.aq_dataset_add_fluid(self._h, fluid._h, pcg_rel_tol, pcg_max_iter, ct.byref(it)))
        return it.value

    def target_rms(self, first: int = 0, count: int = None) -> float:
        v = ct.c_double()
        _check(self._lib.aq_dataset_target_rms(self._h, first, len(self) - first if count is None else count,
                                               ct.byref(v)))
        return v.value

    def get(self, i: int) -> dict:
        n = self.size[0] * self.size[1] * self.size[2]
        rhs, typ, tgt = np.zeros(n, np.float32), np.zeros(n, np.int8), np.zeros(n, np.float32)
        _check(self._lib.aq_dataset_get(self._h, i, rhs.ctypes.data, typ.ctypes.data, tgt.ctypes.data))
        return {"rhs": rhs, "type": typ, "target": tgt}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.aq_dataset_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
