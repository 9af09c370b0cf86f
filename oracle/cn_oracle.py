"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (oracle/cn_oracle.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module; the
product never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libcn_oracle.so"
# The same restatement with the shaders' own quotients in the fluid kernels (no reciprocal
# products); compared bit for bit with the reference's kernels executed on the host.
LIB_QUOTIENTS = HERE / "libcn_oracle_quot.so"

DEBUG = {"cell_entries": 0, "sorted_keys": 1, "cell_ranges": 2, "fluid_neighbor_counts": 3,
         "fluid_neighbors": 4, "fluid_constraints": 5, "fluid_delta": 6, "rigid_contacts": 7}

_libs: dict = {}


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE), "all", "quotients"], check=True)
    return LIB


def load(quotients: bool = False) -> C.CDLL:
    path = LIB_QUOTIENTS if quotients else LIB
    if path not in _libs:
        if not path.exists():
            build()
        lib = C.CDLL(str(path))
        lib.cno_create.restype = C.c_void_p
        lib.cno_create.argtypes = [C.c_void_p, C.c_void_p]
        lib.cno_destroy.argtypes = [C.c_void_p]
        lib.cno_step.argtypes = [C.c_void_p, C.c_float]
        lib.cno_read_particles.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.cno_read_strand_orientations.argtypes = [C.c_void_p, C.c_void_p]
        lib.cno_debug_read.restype = C.c_size_t
        lib.cno_debug_read.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
        lib.cno_set_kinematic_target.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        lib.cno_set_threads.argtypes = [C.c_int]
        lib.cno_set_post_update_neighbors.argtypes = [C.c_void_p, C.c_int]
        lib.cno_meta.restype = C.c_uint32
        lib.cno_meta.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        lib.cno_fluid_material.argtypes = [C.c_float] * 7 + [C.c_void_p]
        lib.cno_read_surface_render.argtypes = [C.c_void_p] * 5
        lib.cno_read_rigid_bodies.argtypes = [C.c_void_p] * 5
        _libs[path] = lib
    return _libs[path]


def set_threads(n: int) -> int:
    return load().cno_set_threads(n)


class Oracle:
    """CPU restatement of PhysicsSolver::step over the same SoA the GPU solver receives."""

    def __init__(self, desc, soa, quotients: bool = False):
        self._lib = load(quotients)
        self._h = self._lib.cno_create(C.byref(desc), C.byref(soa))
        if not self._h:
            raise RuntimeError("oracle: create failed")
        self.n = soa.particle_count
        self.segments = soa.strand_segment_count
        self.bodies = soa.rigid_body_count
        sr = soa.surface_render
        self.surface = (sr.contents.vertex_count, sr.contents.triangle_count, sr.contents.surface_count) if sr \
            else (0, 0, 0)

    def close(self):
        if self._h:
            self._lib.cno_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_post_update_neighbors(self, enable: bool) -> None:
        self._lib.cno_set_post_update_neighbors(self._h, int(enable))

    def step(self, dt: float) -> None:
        self._lib.cno_step(self._h, dt)

    def set_kinematic_target(self, body, position, orientation=(0, 0, 0, 1)):
        p = (C.c_float * 3)(*position)
        q = (C.c_float * 4)(*orientation)
        self._lib.cno_set_kinematic_target(self._h, body, p, q)

    def read_particles(self):
        x = np.zeros((self.n, 4), np.float32)
        v = np.zeros((self.n, 4), np.float32)
        xp = np.zeros((self.n, 4), np.float32)
        self._lib.cno_read_particles(self._h, x.ctypes.data, v.ctypes.data, xp.ctypes.data)
        return x, v, xp

    def read_strand_orientations(self):
        q = np.zeros((self.segments, 4), np.float32)
        if self.segments:
            self._lib.cno_read_strand_orientations(self._h, q.ctypes.data)
        return q

    def read_rigid_bodies(self):
        """(positions with inverse mass, orientations, linear, angular velocities), each (B, 4)."""
        out = [np.zeros((self.bodies, 4), np.float32) for _ in range(4)]
        self._lib.cno_read_rigid_bodies(self._h, *(a.ctypes.data for a in out))
        return tuple(out)

    def read_surface_render(self):
        """(render positions V x 4, render normals V x 4, world AABBs S x 8, triangle normals T x 4)."""
        V, T, S = self.surface
        pos = np.zeros((V, 4), np.float32)
        nrm = np.zeros((V, 4), np.float32)
        box = np.zeros((S, 8), np.float32)
        tri = np.zeros((T, 4), np.float32)
        self._lib.cno_read_surface_render(self._h, pos.ctypes.data, nrm.ctypes.data, box.ctypes.data, tri.ctypes.data)
        return pos, nrm, box, tri

    def debug_read(self, name: str) -> np.ndarray:
        which = DEBUG[name]
        n = self._lib.cno_debug_read(self._h, which, None, 0)
        buf = np.zeros(n, np.uint8)
        if n:
            self._lib.cno_debug_read(self._h, which, buf.ctypes.data, n)
        return buf

    def meta(self) -> dict:
        out = (C.c_uint32 * 11)()
        self._lib.cno_meta(self._h, out, 11)
        keys = ["required_rigid_pairs", "rigid_pairs", "required_particle_pairs", "particle_pairs",
                "active_rigid_contacts", "active_particle_contacts", "neighbor_truncations",
                "required_rigid_rigid_pairs", "rigid_rigid_pairs", "required_proxy_contacts", "proxy_contacts"]
        return dict(zip(keys, list(out)))


def fluid_material(radius, viscosity=0.01, cohesion=0.0, surface_tension=0.0, vorticity=0.0,
                   gravity_scale=1.0, cfl=1.0) -> np.ndarray:
    out = (C.c_float * 12)()
    load().cno_fluid_material(radius, viscosity, cohesion, surface_tension, vorticity, gravity_scale, cfl, out)
    return np.array(list(out), np.float32)
