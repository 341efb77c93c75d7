"""ctypes bindings of the two checkers, for tests only.

* ``Oracle``: the CPU restatement, oracle/liborc.so (flip_oracle.c).
* ``RefFluid``: the reference's own kernels built headless, oracle/_ref/libaqref.so
  (needs a GPU; present only where oracle/Makefile's ``ref`` target was built).
* ``RefMesher``: the reference's own surface mesher, oracle/_ref/libaqmesh.so
  (target ``mesh``; needs a GPU).
* ``RenderOracle``: the CPU restatement of the headless frame (render_oracle.c).
"""
from __future__ import annotations

import ctypes as ct
import os
import pathlib
import subprocess

import numpy as np

from aquarius_b200 import _abi

ROOT = pathlib.Path(__file__).resolve().parent.parent
ORACLE_SO = ROOT / "oracle" / "liborc.so"
REF_SO = ROOT / "oracle" / "_ref" / "libaqref.so"
MESH_SO = ROOT / "oracle" / "_ref" / "libaqmesh.so"
SPH_SO = ROOT / "oracle" / "_ref" / "libaqsph.so"

_orc = None
_ref = None
_mesh = None
_sph = None


def _load_oracle():
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
        lib = ct.CDLL(str(ORACLE_SO))
        lib.orc_create.restype = ct.c_void_p
        lib.orc_create.argtypes = [ct.POINTER(_abi.Config)]
        lib.orc_destroy.argtypes = [ct.c_void_p]
        lib.orc_particle_count.restype = ct.c_int
        lib.orc_particle_count.argtypes = [ct.c_void_p]
        lib.orc_run_stage.restype = ct.c_int
        lib.orc_run_stage.argtypes = [ct.c_void_p, ct.c_int]
        lib.orc_step.restype = ct.c_int
        lib.orc_step.argtypes = [ct.c_void_p, ct.c_int]
        lib.orc_get_state.restype = ct.c_int
        lib.orc_get_state.argtypes = [ct.c_void_p, ct.POINTER(_abi.HostState)]
        lib.orc_set_state.restype = ct.c_int
        lib.orc_set_state.argtypes = [ct.c_void_p, ct.POINTER(_abi.HostState)]
        lib.orc_solve_stats.argtypes = [ct.c_void_p, ct.POINTER(ct.c_int), ct.POINTER(ct.c_double),
                                        ct.POINTER(ct.c_double), ct.POINTER(ct.c_int)]
        lib.orc_set_schedule.argtypes = [ct.c_void_p, ct.c_int]
        lib.orc_pressure_residual.restype = ct.c_double
        lib.orc_pressure_residual.argtypes = [ct.c_void_p]
        lib.orc_threads.restype = ct.c_int
        lib.orc_ink_create.restype = ct.c_int
        lib.orc_ink_create.argtypes = [ct.c_void_p]
        lib.orc_ink_count.restype = ct.c_int
        lib.orc_ink_count.argtypes = [ct.c_void_p]
        lib.orc_ink_advance.argtypes = [ct.c_void_p]
        lib.orc_ink_get.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p]
        lib.orc_ink_set.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p]
        lib.orc_mesh_dims_of.argtypes = [ct.c_void_p, ct.c_void_p]
        lib.orc_sph_create.restype = ct.c_void_p
        lib.orc_sph_create.argtypes = [ct.POINTER(_abi.SphConfig)]
        lib.orc_sph_destroy.argtypes = [ct.c_void_p]
        lib.orc_sph_count.restype = ct.c_int
        lib.orc_sph_count.argtypes = [ct.c_void_p]
        lib.orc_sph_info.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
        lib.orc_sph_step.restype = ct.c_int
        lib.orc_sph_step.argtypes = [ct.c_void_p, ct.c_int]
        lib.orc_sph_get.restype = ct.c_int
        lib.orc_sph_get.argtypes = [ct.c_void_p, ct.POINTER(_abi.SphState)]
        lib.orc_sph_set.restype = ct.c_int
        lib.orc_sph_set.argtypes = [ct.c_void_p, ct.POINTER(_abi.SphState)]
        lib.orc_tex_linear.argtypes = [ct.c_void_p, ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int]
        lib.orc_mesh.restype = ct.c_int
        lib.orc_mesh.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_longlong, ct.POINTER(ct.c_int)]
        P = ct.c_void_p
        lib.orc_render_frame.restype = ct.c_int
        lib.orc_render_frame.argtypes = [P, P, ct.c_int32, P, ct.c_int64, P, ct.c_int32, P, ct.c_int32, ct.c_int32,
                                         P, P]
        lib.orc_trace_environment.argtypes = [P, P, ct.c_int32, P, ct.c_int32, ct.c_int32, P, P, P]
        lib.orc_shade_mesh.argtypes = [P, P, ct.c_int32, P, ct.c_int32, ct.c_int32, P, P, P, P]
        lib.orc_sample_cube.argtypes = [P, ct.c_int32, P, P]
        lib.orc_sample_2d.argtypes = [P, ct.c_int32, ct.c_int32, ct.c_float, ct.c_float, P]
        lib.orc_draw_command_default.argtypes = [P, ct.c_int32, ct.c_int32, ct.c_float, ct.c_int32]
        _orc = lib
    return _orc


def _load_ref():
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            raise FileNotFoundError(str(REF_SO))
        lib = ct.CDLL(str(REF_SO))
        lib.aqref_create.restype = ct.c_void_p
        lib.aqref_create.argtypes = [ct.POINTER(_abi.Config)]
        lib.aqref_destroy.argtypes = [ct.c_void_p]
        lib.aqref_particle_count.restype = ct.c_int
        lib.aqref_particle_count.argtypes = [ct.c_void_p]
        lib.aqref_step.restype = ct.c_int
        lib.aqref_step.argtypes = [ct.c_void_p, ct.c_int]
        lib.aqref_time_steps.restype = ct.c_int
        lib.aqref_time_steps.argtypes = [ct.c_void_p, ct.c_int, ct.POINTER(ct.c_float)]
        lib.aqref_stage.restype = ct.c_int
        lib.aqref_stage.argtypes = [ct.c_void_p, ct.c_int]
        lib.aqref_get_state.restype = ct.c_int
        lib.aqref_get_state.argtypes = [ct.c_void_p, ct.POINTER(_abi.HostState)]
        lib.aqref_set_state.restype = ct.c_int
        lib.aqref_set_state.argtypes = [ct.c_void_p, ct.POINTER(_abi.HostState)]
        lib.aqref_probe_texture.restype = ct.c_int
        lib.aqref_probe_texture.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_int]
        lib.aqref_error.restype = ct.c_int
        lib.aqref_ink_init.restype = ct.c_int
        lib.aqref_ink_init.argtypes = [ct.c_void_p]
        for nm in ("aqref_ink_step",):
            getattr(lib, nm).restype = ct.c_int
            getattr(lib, nm).argtypes = [ct.c_void_p]
        for nm in ("aqref_ink_get", "aqref_ink_set"):
            getattr(lib, nm).restype = ct.c_int
            getattr(lib, nm).argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p]
        _ref = lib
    return _ref


def ref_available() -> bool:
    return REF_SO.exists()


def mesh_ref_available() -> bool:
    return MESH_SO.exists()


def _load_mesh():
    global _mesh
    if _mesh is None:
        if not MESH_SO.exists():
            raise FileNotFoundError(str(MESH_SO))
        lib = ct.CDLL(str(MESH_SO))
        lib.aqmesh_create.restype = ct.c_void_p
        lib.aqmesh_create.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_float, ct.c_int]
        lib.aqmesh_destroy.argtypes = [ct.c_void_p]
        lib.aqmesh_sizes.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
        lib.aqmesh_run.restype = ct.c_int
        lib.aqmesh_run.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_longlong, ct.POINTER(ct.c_int),
                                   ct.c_void_p, ct.c_void_p, ct.POINTER(ct.c_float)]
        lib.aqmesh_probe_linear.restype = ct.c_int
        lib.aqmesh_probe_linear.argtypes = [ct.c_int, ct.c_int, ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                            ct.c_int]
        lib.aqmesh_error.restype = ct.c_int
        _mesh = lib
    return _mesh


class RefMesher:
    """The reference's Mesher (Rendering/Renderer3D/Mesher.cu) on the GPU,
    built as Fluid::init builds it for an sx*sy*sz grid of cell size h."""

    def __init__(self, size, h: float, n: int):
        self.lib = _load_mesh()
        self.n = n
        self.h = self.lib.aqmesh_create(size[0], size[1], size[2], h, n)
        if not self.h:
            raise RuntimeError(f"reference mesher init failed: {self.lib.aqmesh_error()}")
        sdf = (ct.c_int * 3)()
        mesh = (ct.c_int * 3)()
        cell = (ct.c_float * 2)()
        self.lib.aqmesh_sizes(self.h, sdf, mesh, cell)
        self.sdf_size = tuple(sdf)
        self.mesh_size = tuple(mesh)
        self.h_sdf, self.h_mesh = cell[0], cell[1]

    def mesh(self, position: np.ndarray, capacity_cubes: int = 1 << 18, want_sdf=True, want_order=False) -> dict:
        pos = np.ascontiguousarray(position, np.float32).reshape(3, self.n)
        out = np.zeros(capacity_cubes * 90, np.float32)
        cubes = ct.c_int()
        sx, sy, sz = self.sdf_size
        sdf = np.zeros(sx * sy * sz, np.float32) if want_sdf else None
        after = np.zeros((3, self.n), np.float32) if want_order else None
        ms = ct.c_float()
        rc = self.lib.aqmesh_run(self.h, pos.ctypes.data, out.ctypes.data, out.size, ct.byref(cubes),
                                 None if sdf is None else sdf.ctypes.data, None if after is None else after.ctypes.data,
                                 ct.byref(ms))
        if rc != 0:
            raise RuntimeError(f"reference mesh failed: {rc}")
        res = {"cubes": cubes.value, "records": out[: min(cubes.value, capacity_cubes) * 90].reshape(-1, 15, 6),
               "ms": ms.value}
        if sdf is not None:
            res["sdf"] = sdf.reshape(sz, sy, sx)  # x fastest
        if after is not None:
            res["position_after"] = after
        return res

    def close(self):
        if self.h:
            self.lib.aqmesh_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def probe_linear(values: np.ndarray, coords) -> np.ndarray:
    """Reads a [d, h, w] float field through the reference's linear-filtered,
    x-border texture (the mesher's SDF settings) at coords ([k, 3], x y z)."""
    lib = _load_mesh()
    v = np.ascontiguousarray(values, np.float32)
    d, h, w = v.shape
    c = np.ascontiguousarray(np.asarray(coords, dtype=np.float32))
    out = np.zeros(len(c), np.float32)
    rc = lib.aqmesh_probe_linear(w, h, d, v.ctypes.data, c.ctypes.data, out.ctypes.data, len(c))
    if rc != 0:
        raise RuntimeError(f"probe failed {rc}")
    return out


class _InkIO:
    """Ink particles over [3, n] numpy planes, shared by both checkers."""

    n_ink: int = 0

    def get_ink(self) -> dict:
        pos = np.zeros((3, self.n_ink), np.float32)
        vel = np.zeros((3, self.n_ink), np.float32)
        rc = self._ink_get(pos.ctypes.data, vel.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"ink get failed: {rc}")
        return {"position": pos, "velocity": vel}

    def set_ink(self, position=None, velocity=None):
        p = None if position is None else np.ascontiguousarray(position, np.float32).reshape(3, self.n_ink)
        v = None if velocity is None else np.ascontiguousarray(velocity, np.float32).reshape(3, self.n_ink)
        rc = self._ink_set(None if p is None else p.ctypes.data, None if v is None else v.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"ink set failed: {rc}")


class _StateIO(_InkIO):
    """get_state/set_state over numpy dicts, shared by both checkers."""

    size: tuple
    n: int

    def get_state(self, fields=None) -> dict:
        sx, sy, sz = self.size
        arrs = _abi.alloc_state(sx, sy, sz, self.n, fields)
        st = _abi.make_host_state(sx, sy, sz, self.n, arrs)
        rc = self._get(ct.byref(st))
        if rc != 0:
            raise RuntimeError(f"get_state failed: {rc}")
        arrs["physical_time"] = st.physical_time
        return arrs

    def set_state(self, state: dict):
        sx, sy, sz = self.size
        arrs = {k: np.ascontiguousarray(v) for k, v in state.items() if k in _abi.STATE_FIELDS}
        st = _abi.make_host_state(sx, sy, sz, self.n, arrs, float(state.get("physical_time", 0.0)))
        rc = self._set(ct.byref(st))
        if rc != 0:
            raise RuntimeError(f"set_state failed: {rc}")


class Oracle(_StateIO):
    """CPU restatement of the reference step (test infrastructure)."""

    def __init__(self, cfg: _abi.Config):
        self.lib = _load_oracle()
        self.cfg = cfg
        self.h = self.lib.orc_create(ct.byref(cfg))
        if not self.h:
            raise ValueError("oracle rejected the config")
        self.size = (cfg.size_x, cfg.size_y, cfg.size_z)
        self.n = self.lib.orc_particle_count(self.h)

    def _get(self, p):
        return self.lib.orc_get_state(self.h, p)

    def _set(self, p):
        return self.lib.orc_set_state(self.h, p)

    def stage(self, k: int):
        if self.lib.orc_run_stage(self.h, k) != 0:
            raise RuntimeError("bad stage")

    def step(self, n: int = 1):
        if self.lib.orc_step(self.h, n) != 0:
            raise RuntimeError("step failed")

    def solve_stats(self):
        it, nf = ct.c_int(), ct.c_int()
        rr, bn = ct.c_double(), ct.c_double()
        self.lib.orc_solve_stats(self.h, ct.byref(it), ct.byref(rr), ct.byref(bn), ct.byref(nf))
        return {"iterations": it.value, "rel_residual": rr.value, "b_norm": bn.value, "fluid_cells": nf.value}

    def pressure_residual(self) -> float:
        return self.lib.orc_pressure_residual(self.h)

    def set_schedule(self, serial: bool):
        """serial: the in-place Jacobi / extrapolation in a serial schedule of
        the reference's launch instead of the race-free reading."""
        self.lib.orc_set_schedule(self.h, 1 if serial else 0)

    def mesh_dims(self) -> dict:
        buf = (ct.c_byte * 64)()  # orc_mesh_dims: int sdf[3], mesh[3]; float h_sdf, h_mesh, radius
        self.lib.orc_mesh_dims_of(self.h, buf)
        ints = np.frombuffer(bytes(buf)[:24], np.int32)
        fl = np.frombuffer(bytes(buf)[24:36], np.float32)
        return {"sdf": tuple(int(v) for v in ints[:3]), "mesh": tuple(int(v) for v in ints[3:6]),
                "h_sdf": float(fl[0]), "h_mesh": float(fl[1]), "radius": float(fl[2])}

    def mesh(self) -> dict:
        """SDF grid ([x][y][z]) and the occupied-cube records ([k, 15, 6])."""
        d = self.mesh_dims()
        cubes = ct.c_int()
        self.lib.orc_mesh(self.h, None, None, 0, ct.byref(cubes))
        sdf = np.zeros(d["sdf"], np.float32)
        rec = np.zeros((max(cubes.value, 1), 15, 6), np.float32)
        if self.lib.orc_mesh(self.h, sdf.ctypes.data, rec.ctypes.data, cubes.value, ct.byref(cubes)) != 0:
            raise MemoryError("oracle mesh")
        return {"sdf": sdf, "records": rec[: cubes.value], "cubes": cubes.value, "dims": d}

    def enable_ink(self) -> int:
        self.n_ink = self.lib.orc_ink_create(self.h)
        return self.n_ink

    def ink_advance(self):
        self.lib.orc_ink_advance(self.h)

    def _ink_get(self, p, v):
        self.lib.orc_ink_get(self.h, p, v)
        return 0

    def _ink_set(self, p, v):
        self.lib.orc_ink_set(self.h, p, v)
        return 0

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefFluid(_StateIO):
    """The reference's Fluid_3D_FLIP::Fluid on the GPU (test infrastructure)."""

    def __init__(self, cfg: _abi.Config):
        self.lib = _load_ref()
        self.h = self.lib.aqref_create(ct.byref(cfg))
        if not self.h:
            raise RuntimeError(f"reference init failed: cuda error {self.lib.aqref_error()}")
        self.size = (cfg.size_x, cfg.size_y, cfg.size_z)
        self.n = self.lib.aqref_particle_count(self.h)

    def _get(self, p):
        return self.lib.aqref_get_state(self.h, p)

    def _set(self, p):
        return self.lib.aqref_set_state(self.h, p)

    def stage(self, k: int):
        rc = self.lib.aqref_stage(self.h, k)
        if rc != 0:
            raise RuntimeError(f"reference stage {k} failed: {rc}")

    def step(self, n: int = 1):
        rc = self.lib.aqref_step(self.h, n)
        if rc != 0:
            raise RuntimeError(f"reference step failed: {rc}")

    def time_steps(self, n: int) -> float:
        """Milliseconds of n simulationStep()s, CUDA events on the legacy
        default stream (the reference's own device syncs included)."""
        ms = ct.c_float()
        rc = self.lib.aqref_time_steps(self.h, n, ct.byref(ms))
        if rc != 0:
            raise RuntimeError(f"reference step failed: {rc}")
        return float(ms.value)

    def enable_ink(self) -> int:
        n = self.lib.aqref_ink_init(self.h)
        if n < 0:
            raise RuntimeError(f"reference ink init failed: {self.lib.aqref_error()}")
        self.n_ink = n
        return n

    def ink_advance(self):
        rc = self.lib.aqref_ink_step(self.h)
        if rc != 0:
            raise RuntimeError(f"reference ink step failed: {rc}")

    def _ink_get(self, p, v):
        return self.lib.aqref_ink_get(self.h, p, v)

    def _ink_set(self, p, v):
        return self.lib.aqref_ink_set(self.h, p, v)

    def close(self):
        if self.h:
            self.lib.aqref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def probe_texture(w, h, d, coords) -> np.ndarray:
    """Reads the reference's createField3D<float> texture at coords ([k,3])."""
    lib = _load_ref()
    c = np.ascontiguousarray(np.asarray(coords, dtype=np.float32))
    out = np.zeros(len(c), dtype=np.float32)
    rc = lib.aqref_probe_texture(w, h, d, c.ctypes.data, out.ctypes.data, len(c))
    if rc != 0:
        raise RuntimeError(f"probe failed {rc}")
    return out


def oracle_threads() -> int:
    return _load_oracle().orc_threads()


def oracle_tex_linear(values: np.ndarray, coords) -> np.ndarray:
    """The oracle's model of the linear-filtered, x-border texture on a
    [d, h, w] field (as probe_linear takes it) at coords ([k, 3], x y z)."""
    lib = _load_oracle()
    v = np.ascontiguousarray(np.asarray(values, np.float32).transpose(2, 1, 0))  # -> [w][h][d], z fastest
    w, h, d = v.shape
    c = np.ascontiguousarray(np.asarray(coords, dtype=np.float32))
    out = np.zeros(len(c), np.float32)
    lib.orc_tex_linear(v.ctypes.data, w, h, d, c.ctypes.data, out.ctypes.data, len(c))
    return out


class _SphStateIO:
    """aq_sph_state exchange over numpy dicts, shared by the SPH checkers."""

    n: int

    def get_state(self, fields=None) -> dict:
        arrs = _abi.alloc_sph_state(self.n, fields)
        st = _abi.make_sph_state(self.n, arrs)
        rc = self._get(ct.byref(st))
        if rc != 0:
            raise RuntimeError(f"get_state failed: {rc}")
        arrs["physical_time"] = st.physical_time
        return arrs

    def set_state(self, state: dict):
        arrs = {k: np.ascontiguousarray(v, np.float32) for k, v in state.items() if k in _abi.SPH_FIELDS}
        st = _abi.make_sph_state(self.n, arrs, float(state.get("physical_time", 0.0)))
        rc = self._set(ct.byref(st))
        if rc != 0:
            raise RuntimeError(f"set_state failed: {rc}")


class SphOracle(_SphStateIO):
    """CPU restatement of the reference's PBF / PCISPH solvers (test infrastructure)."""

    def __init__(self, cfg: _abi.SphConfig):
        self.lib = _load_oracle()
        self.cfg = cfg
        self.h = self.lib.orc_sph_create(ct.byref(cfg))
        if not self.h:
            raise ValueError("oracle rejected the config")
        self.n = self.lib.orc_sph_count(self.h)
        sp, kr = ct.c_float(), ct.c_float()
        g = (ct.c_int * 3)()
        self.lib.orc_sph_info(self.h, ct.byref(sp), ct.byref(kr), g)
        self.spacing, self.kernel_radius, self.grid = sp.value, kr.value, tuple(g)

    def _get(self, p):
        return self.lib.orc_sph_get(self.h, p)

    def _set(self, p):
        return self.lib.orc_sph_set(self.h, p)

    def step(self, n: int = 1):
        self.lib.orc_sph_step(self.h, n)

    def close(self):
        if self.h:
            self.lib.orc_sph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sph_ref_available() -> bool:
    return SPH_SO.exists()


def _load_sph():
    global _sph
    if _sph is None:
        if not SPH_SO.exists():
            raise FileNotFoundError(str(SPH_SO))
        lib = ct.CDLL(str(SPH_SO))
        lib.aqsph_create.restype = ct.c_void_p
        lib.aqsph_create.argtypes = [ct.POINTER(_abi.SphConfig)]
        lib.aqsph_destroy.argtypes = [ct.c_void_p]
        lib.aqsph_count.restype = ct.c_int
        lib.aqsph_count.argtypes = [ct.c_void_p]
        lib.aqsph_error.restype = ct.c_int
        lib.aqsph_step.restype = ct.c_int
        lib.aqsph_step.argtypes = [ct.c_void_p, ct.c_int]
        lib.aqsph_get.restype = ct.c_int
        lib.aqsph_get.argtypes = [ct.c_void_p, ct.POINTER(_abi.SphState)]
        lib.aqsph_set.restype = ct.c_int
        lib.aqsph_set.argtypes = [ct.c_void_p, ct.POINTER(_abi.SphState)]
        lib.aqsph_info.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
        _sph = lib
    return _sph


class RefSph(_SphStateIO):
    """The reference's Fluid_3D_PBF / Fluid_3D_PCISPH::Fluid on the GPU (test infrastructure)."""

    def __init__(self, cfg: _abi.SphConfig):
        self.lib = _load_sph()
        self.h = self.lib.aqsph_create(ct.byref(cfg))
        if not self.h:
            raise RuntimeError(f"reference init failed: cuda error {self.lib.aqsph_error()}")
        self.n = self.lib.aqsph_count(self.h)
        sp, kr = ct.c_float(), ct.c_float()
        g = (ct.c_int * 3)()
        self.lib.aqsph_info(self.h, ct.byref(sp), ct.byref(kr), g)
        self.spacing, self.kernel_radius, self.grid = sp.value, kr.value, tuple(g)

    def _get(self, p):
        return self.lib.aqsph_get(self.h, p)

    def _set(self, p):
        return self.lib.aqsph_set(self.h, p)

    def step(self, n: int = 1):
        rc = self.lib.aqsph_step(self.h, n)
        if rc != 0:
            raise RuntimeError(f"reference step failed: {rc}")

    def close(self):
        if self.h:
            self.lib.aqsph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(a):
    return None if a is None else a.ctypes.data


class RenderOracle:
    """render_oracle.c: one frame drawn GL-style on the CPU (test infrastructure)."""

    def __init__(self, sky=None, logo=None):
        self.lib = _load_oracle()
        self.sky = None if sky is None else np.ascontiguousarray(sky, np.uint8)
        self.logo = None if logo is None else np.ascontiguousarray(logo, np.uint8)
        self.face = 0 if self.sky is None else int(self.sky.shape[1])
        self.lw = 0 if self.logo is None else int(self.logo.shape[1])
        self.lh = 0 if self.logo is None else int(self.logo.shape[0])

    def frame(self, dc, points=None, mesh=None):
        """points: float32 [N, 7]; mesh: float32 [V, 6].  Returns (rgba [H, W, 4], phase [H, W, 4])."""
        h, w = dc.window_height, dc.window_width
        rgba = np.zeros((h, w, 4), np.uint8)
        phase = np.zeros((h, w, 4), np.float32)
        pts = None if points is None else np.ascontiguousarray(points, np.float32).reshape(-1, 7)
        msh = None if mesh is None else np.ascontiguousarray(mesh, np.float32).reshape(-1, 6)
        rc = self.lib.orc_render_frame(ct.byref(dc), _ptr(pts), 0 if pts is None else pts.shape[0], _ptr(msh),
                                       0 if msh is None else msh.shape[0], _ptr(self.sky), self.face,
                                       _ptr(self.logo), self.lw, self.lh, rgba.ctypes.data, phase.ctypes.data)
        if rc != 0:
            raise ValueError("orc_render_frame rejected its arguments")
        return rgba, phase

    def trace(self, dc, origin, direction):
        o = np.ascontiguousarray(origin, np.float32)
        d = np.ascontiguousarray(direction, np.float32)
        out = np.zeros(4, np.float32)
        self.lib.orc_trace_environment(ct.byref(dc), _ptr(self.sky), self.face, _ptr(self.logo), self.lw, self.lh,
                                       o.ctypes.data, d.ctypes.data, out.ctypes.data)
        return out

    def shade_mesh(self, dc, frag_pos, frag_normal, texel):
        p = np.ascontiguousarray(frag_pos, np.float32)
        n = np.ascontiguousarray(frag_normal, np.float32)
        t = np.ascontiguousarray(texel, np.float32)
        out = np.zeros(4, np.float32)
        self.lib.orc_shade_mesh(ct.byref(dc), _ptr(self.sky), self.face, _ptr(self.logo), self.lw, self.lh,
                                p.ctypes.data, n.ctypes.data, t.ctypes.data, out.ctypes.data)
        return out

    @staticmethod
    def draw_command_default(width, height, domain_size, size_y):
        dc = _abi.DrawCommand()
        _load_oracle().orc_draw_command_default(ct.byref(dc), int(width), int(height), float(domain_size),
                                                int(size_y))
        return dc
