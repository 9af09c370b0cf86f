"""Python host mirror of the CRESSim-Neo particle substep (B200 build).

The classes follow the reference's host API for this path:

* ``World``  -- PhysicsWorld authoring (upsertSoftBody / fluids / cloth / strands / rigid bodies and
  colliders, reference include/physics/physics_world.h) producing the particle/constraint SoA;
* ``Solver`` -- PhysicsSolver (include/physics/physics_solver.h:150-205): ``sync_world``,
  ``step``, ``validate_gpu_meta``, ``set_gravity``, ``gpu_scene_view``.

Everything runs through the C ABI of ``libcn_physics.so`` (include/cn_physics.h); there is no
Python or CPU implementation of the substep in this package.
"""
from __future__ import annotations

import ctypes as C
import weakref
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import load

__all__ = ["World", "Solver", "SolverDesc", "CNError", "load", "solver_desc", "DEBUG"]

STATUS = {0: "OK", 1: "INVALID_ARGUMENT", 2: "CUDA", 3: "OUT_OF_MEMORY", 4: "NOT_INITIALIZED",
          5: "CAPACITY", 6: "NO_DEVICE", 7: "DEVICE_TIMEOUT", 8: "UNSUPPORTED"}

DEBUG = {"cell_entries": 0, "sorted_keys": 1, "cell_ranges": 2, "fluid_neighbor_counts": 3,
         "fluid_neighbors": 4, "fluid_constraints": 5, "fluid_delta": 6, "rigid_contacts": 7,
         "fluid_superset_counts": 8}

SolverDesc = _abi.SolverDesc


class CNError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


def _check(status: int) -> None:
    if status != 0:
        raise CNError(status, load().cn_last_error().decode())


def solver_desc(**overrides) -> _abi.SolverDesc:
    """PhysicsSolverDesc with the reference defaults (physics_solver.h:22-143), then overrides.

    Nested settings may be given as ``contact_slop=...``, ``soft_internal_relaxation=...``,
    ``fluid_constraint_relaxation=...``; ``gravity=(x, y, z)``."""
    d = _abi.SolverDesc()
    load().cn_solver_desc_defaults(C.byref(d))
    for key, value in overrides.items():
        if key == "gravity":
            d.gravity = (C.c_float * 3)(*value)
        elif hasattr(d, key):
            setattr(d, key, value)
        else:
            group, _, name = key.partition("_")
            setattr(getattr(d, group), name, value)
    return d


def colour_constraints(elements, element_count: int) -> tuple:
    """Greedy graph colouring of one constraint family (host only): `elements` (M, k) uint32 are
    each constraint's particles (segments for strand joints); entries >= element_count are
    ignored.  Returns (order, starts): the constraints grouped by colour, ascending within a
    colour, and the colour boundaries (colours + 1 entries)."""
    e = np.ascontiguousarray(elements, dtype=np.uint32)
    m = e.shape[0]
    k = e.shape[1] if e.ndim == 2 else 1
    order = np.zeros(max(m, 1), np.uint32)
    cap = max(k * 64, 64)
    while True:
        starts = np.zeros(cap + 1, np.uint32)
        n = C.c_uint32()
        st = load().cn_colour_constraints(e.ctypes.data_as(_abi.P_u32), m, k, element_count,
                                          order.ctypes.data_as(_abi.P_u32), starts.ctypes.data_as(_abi.P_u32),
                                          cap, C.byref(n))
        if st == 0:
            return order[:m].copy(), starts[:n.value + 1].copy()
        if n.value > cap:
            cap = n.value
            continue
        _check(st)


def _f32(arr) -> C.POINTER(C.c_float):
    return arr.ctypes.data_as(_abi.P_f32)


def _u32(arr) -> C.POINTER(C.c_uint32):
    return arr.ctypes.data_as(_abi.P_u32)


def _view(ptr, count: int, dtype, cols: int = 1) -> np.ndarray:
    if count == 0 or not ptr:
        return np.zeros((count, cols) if cols > 1 else (count,), dtype=dtype)
    ctype = C.c_float if dtype == np.float32 else C.c_uint32
    base = C.cast(ptr, C.POINTER(ctype))
    a = np.ctypeslib.as_array(base, shape=(count * cols,))
    return a.reshape(count, cols) if cols > 1 else a


class World:
    """PhysicsWorld authoring mirror.  ``soa()`` packs the SoA the solver uploads; the position and
    velocity arrays it exposes are views that may be edited in place before ``sync_world``."""

    def __init__(self):
        self._lib = load()
        h = C.c_void_p()
        _check(self._lib.cn_world_create(C.byref(h)))
        self._h = h
        self._soa: Optional[_abi.WorldSoA] = None
        self._keep = []

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cn_world_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _transform(t, position=(0, 0, 0), rotation=(0, 0, 0, 1), scale=(1, 1, 1)):
        t.position = (C.c_float * 3)(*position)
        t.rotation = (C.c_float * 4)(*rotation)
        t.scale = (C.c_float * 3)(*scale)

    @staticmethod
    def _material(m, friction=0.0, restitution=0.0, damping=0.0, static_friction=-1.0):
        m.friction, m.restitution, m.damping, m.static_friction = friction, restitution, damping, static_friction

    def add_soft_body_grid(self, size, spacing, position=(0, 0, 0), rotation=(0, 0, 0, 1), *, mass=1.0,
                           radius=0.125, edge_compliance=0.0, volume_compliance=0.0, self_collision=False,
                           static_particles: Sequence[int] = (), environment=0, layer=1, mask=0xFFFFFFFF,
                           friction=0.0, restitution=0.0, damping=0.0, static_friction=-1.0) -> int:
        """SoftBodyState with a RegularGrid source (soft_body_authoring.cpp:81-176)."""
        d = self._soft_desc(position, rotation, mass, radius, edge_compliance, volume_compliance, self_collision,
                            static_particles, environment, layer, mask, friction, restitution, damping,
                            static_friction)
        d.size = (C.c_float * 3)(*size)
        d.target_particle_spacing = spacing
        out = C.c_uint32()
        _check(self._lib.cn_world_add_soft_body_grid(self._h, C.byref(d), C.byref(out)))
        return out.value

    def add_soft_body_tet_mesh(self, positions, tets, position=(0, 0, 0), rotation=(0, 0, 0, 1), **kw) -> int:
        """SoftBodyState with a TetMesh source: object-space (V, 3) positions, (T, 4) indices."""
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float32).reshape(-1, 3))
        idx = np.ascontiguousarray(np.asarray(tets, dtype=np.uint32).reshape(-1, 4))
        d = self._soft_desc(position, rotation, **self._soft_kw(kw))
        out = C.c_uint32()
        _check(self._lib.cn_world_add_soft_body_tet_mesh(self._h, C.byref(d), _f32(pos), pos.shape[0], _u32(idx),
                                                         idx.shape[0], C.byref(out)))
        return out.value

    def add_soft_body_tetgen(self, node_file, ele_file, position=(0, 0, 0), rotation=(0, 0, 0, 1), **kw) -> int:
        """SoftBodyState with a TetGenFiles source (.node / .ele pair)."""
        d = self._soft_desc(position, rotation, **self._soft_kw(kw))
        out = C.c_uint32()
        _check(self._lib.cn_world_add_soft_body_tetgen(self._h, C.byref(d), str(node_file).encode(),
                                                       str(ele_file).encode(), C.byref(out)))
        return out.value

    def add_soft_body_meshfree(self, positions, neighbours, position=(0, 0, 0), rotation=(0, 0, 0, 1), **kw) -> int:
        """SoftBodyState with a MeshfreeParticles source (k-nearest distance graph)."""
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float32).reshape(-1, 3))
        d = self._soft_desc(position, rotation, **self._soft_kw(kw))
        out = C.c_uint32()
        _check(self._lib.cn_world_add_soft_body_meshfree(self._h, C.byref(d), _f32(pos), pos.shape[0], neighbours,
                                                         C.byref(out)))
        return out.value

    @staticmethod
    def _soft_kw(kw):
        names = ("mass", "radius", "edge_compliance", "volume_compliance", "self_collision", "static_particles",
                 "environment", "layer", "mask", "friction", "restitution", "damping", "static_friction")
        defaults = (1.0, 0.125, 0.0, 0.0, False, (), 0, 1, 0xFFFFFFFF, 0.0, 0.0, 0.0, -1.0)
        unknown = set(kw) - set(names)
        if unknown:
            raise TypeError(f"unknown soft body arguments: {sorted(unknown)}")
        return {n: kw.get(n, dv) for n, dv in zip(names, defaults)}

    def _soft_desc(self, position, rotation, mass, radius, edge_compliance, volume_compliance, self_collision,
                   static_particles, environment, layer, mask, friction, restitution, damping, static_friction):
        d = _abi.SoftBodyGridDesc()
        self._lib.cn_soft_body_grid_desc_defaults(C.byref(d))
        self._transform(d.rest_transform, position, rotation)
        d.particle_mass, d.particle_radius = mass, radius
        d.edge_compliance, d.volume_compliance = edge_compliance, volume_compliance
        d.self_collision_enabled = int(self_collision)
        d.environment_index, d.collision_layer, d.collision_mask = environment, layer, mask
        self._material(d.material, friction, restitution, damping, static_friction)
        st = np.ascontiguousarray(np.asarray(static_particles, dtype=np.uint32))
        self._keep.append(st)
        d.static_particle_indices = _u32(st) if st.size else None
        d.static_particle_count = st.size
        return d

    def add_fluid_grid(self, size, spacing, position=(0, 0, 0), *, mass=1.0, radius=0.05, viscosity=0.01,
                       cohesion=0.0, surface_tension=0.0, vorticity=0.0, gravity_scale=1.0, cfl=1.0,
                       environment=0, layer=1, mask=0xFFFFFFFF, friction=0.0, restitution=0.0, damping=0.0,
                       static_friction=-1.0) -> int:
        """FluidState with a RegularGrid source (physics_world.cpp:6857-6891)."""
        d = _abi.FluidGridDesc()
        self._lib.cn_fluid_grid_desc_defaults(C.byref(d))
        d.size = (C.c_float * 3)(*size)
        d.target_particle_spacing = spacing
        self._transform(d.rest_transform, position)
        d.particle_mass, d.particle_radius = mass, radius
        d.viscosity, d.cohesion, d.surface_tension = viscosity, cohesion, surface_tension
        d.vorticity_confinement, d.gravity_scale, d.cfl_coefficient = vorticity, gravity_scale, cfl
        d.environment_index, d.collision_layer, d.collision_mask = environment, layer, mask
        self._material(d.material, friction, restitution, damping, static_friction)
        out = C.c_uint32()
        _check(self._lib.cn_world_add_fluid_grid(self._h, C.byref(d), C.byref(out)))
        return out.value

    def add_cloth_grid(self, resolution, size, position=(0, 0, 0), rotation=(0, 0, 0, 1), *, mass=1.0,
                       radius=0.02, structural_compliance=0.0, bend_compliance=0.0, self_collision=False,
                       static_particles: Sequence[int] = (), environment=0, layer=1, mask=0xFFFFFFFF,
                       friction=0.0, restitution=0.0, damping=0.0, static_friction=-1.0) -> int:
        """ClothState over a rectangular triangle grid (cloth_authoring.cpp:58-191)."""
        d = _abi.ClothGridDesc()
        self._lib.cn_cloth_grid_desc_defaults(C.byref(d))
        d.resolution = (C.c_uint32 * 2)(*resolution)
        d.size = (C.c_float * 2)(*size)
        self._transform(d.rest_transform, position, rotation)
        d.particle_mass, d.particle_radius = mass, radius
        d.structural_compliance, d.bend_compliance = structural_compliance, bend_compliance
        d.self_collision_enabled = int(self_collision)
        d.environment_index, d.collision_layer, d.collision_mask = environment, layer, mask
        self._material(d.material, friction, restitution, damping, static_friction)
        st = np.ascontiguousarray(np.asarray(static_particles, dtype=np.uint32))
        self._keep.append(st)
        d.static_particle_indices = _u32(st) if st.size else None
        d.static_particle_count = st.size
        out = C.c_uint32()
        _check(self._lib.cn_world_add_cloth_grid(self._h, C.byref(d), C.byref(out)))
        return out.value

    def add_strand(self, rest_positions, *, mass=1.0, radius=0.01, stretch_shear_compliance=0.0,
                   bend_compliance=0.0, twist_compliance=0.0, distance_compliance=0.0, self_collision=False,
                   static_particles: Sequence[int] = (), environment=0, layer=1, mask=0xFFFFFFFF,
                   friction=0.0, restitution=0.0, damping=0.0, static_friction=-1.0) -> int:
        """StrandState (physics_world.cpp:6893-6969)."""
        d = _abi.StrandDesc()
        self._lib.cn_strand_desc_defaults(C.byref(d))
        pts = np.ascontiguousarray(np.asarray(rest_positions, dtype=np.float32).reshape(-1, 3))
        self._keep.append(pts)
        d.rest_positions = _f32(pts)
        d.rest_position_count = pts.shape[0]
        d.particle_mass, d.particle_radius = mass, radius
        d.stretch_shear_compliance, d.bend_compliance = stretch_shear_compliance, bend_compliance
        d.twist_compliance, d.distance_compliance = twist_compliance, distance_compliance
        d.self_collision_enabled = int(self_collision)
        d.environment_index, d.collision_layer, d.collision_mask = environment, layer, mask
        self._material(d.material, friction, restitution, damping, static_friction)
        st = np.ascontiguousarray(np.asarray(static_particles, dtype=np.uint32))
        self._keep.append(st)
        d.static_particle_indices = _u32(st) if st.size else None
        d.static_particle_count = st.size
        out = C.c_uint32()
        _check(self._lib.cn_world_add_strand(self._h, C.byref(d), C.byref(out)))
        return out.value

    def add_rigid_body(self, body_type="static", position=(0, 0, 0), orientation=(0, 0, 0, 1),
                       scale=(1, 1, 1), *, mass=None, inverse_inertia=None) -> int:
        """RigidBodyState: mass and local inverse inertia matter for dynamic bodies."""
        d = _abi.RigidBodyDesc()
        self._lib.cn_rigid_body_desc_defaults(C.byref(d))
        d.body_type = {"static": 0, "kinematic": 1, "dynamic": 2}[body_type]
        d.position = (C.c_float * 3)(*position)
        d.orientation = (C.c_float * 4)(*orientation)
        d.scale = (C.c_float * 3)(*scale)
        if mass is not None:
            d.mass = mass
        if inverse_inertia is not None:
            d.inverse_inertia_local = (C.c_float * 3)(*inverse_inertia)
        out = C.c_uint32()
        _check(self._lib.cn_world_add_rigid_body(self._h, C.byref(d), C.byref(out)))
        return out.value

    def add_collider(self, body, shape, params, local_position=(0, 0, 0), local_orientation=(0, 0, 0, 1), *,
                     friction=0.5, static_friction=-1.0, restitution=0.0, enabled=True, environment=0,
                     layer=1, mask=0xFFFFFFFF) -> int:
        d = _abi.ColliderDesc()
        self._lib.cn_collider_desc_defaults(C.byref(d))
        d.body = body
        d.shape_type = {"sphere": 0, "box": 1, "capsule": 2}[shape]
        p = list(params) + [0.0] * (4 - len(params))
        d.shape_params = (C.c_float * 4)(*p)
        d.local_position = (C.c_float * 3)(*local_position)
        d.local_orientation = (C.c_float * 4)(*local_orientation)
        d.enabled = int(enabled)
        d.friction, d.static_friction, d.restitution = friction, static_friction, restitution
        d.environment_index, d.collision_layer, d.collision_mask = environment, layer, mask
        out = C.c_uint32()
        _check(self._lib.cn_world_add_collider(self._h, C.byref(d), C.byref(out)))
        return out.value

    def set_rigid_proxy_particles(self, body: int, local_positions, radius: float, *, friction=0.5,
                                  restitution=0.0, damping=0.0, static_friction=-1.0, environment=0, layer=1,
                                  mask=0xFFFFFFFF) -> None:
        """Proxy collision particles of `body` at (K, 3) body-frame points (before the body scale):
        carried with the body, they collide with particles and with other bodies' colliders."""
        pos = np.ascontiguousarray(np.asarray(local_positions, dtype=np.float32).reshape(-1, 3))
        d = _abi.RigidProxyDesc()
        self._lib.cn_rigid_proxy_desc_defaults(C.byref(d))
        d.body = body
        d.local_positions = pos.ctypes.data_as(_abi.P_f32)
        d.count = pos.shape[0]
        d.radius = radius
        d.material = _abi.ContactMaterialDesc(friction, restitution, damping, static_friction)
        d.environment_index, d.collision_layer, d.collision_mask = environment, layer, mask
        _check(self._lib.cn_world_set_rigid_proxy_particles(self._h, C.byref(d)))
        self._soa = None

    def add_surface_mesh(self, owner: str, index: int, positions, indices, normals=None,
                         match_epsilon: float = 1.0e-3) -> int:
        """Binds a render mesh to soft body / cloth `index` (owner "soft_body" or "cloth"): (V, 3)
        positions in the owner's object frame, (F, 3) triangle indices, optional (V, 3) fallback
        normals.  Returns the mesh's first render vertex in the packed render arrays."""
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float32).reshape(-1, 3))
        idx = np.ascontiguousarray(np.asarray(indices, dtype=np.uint32).reshape(-1))
        nrm = None if normals is None else np.ascontiguousarray(np.asarray(normals, dtype=np.float32).reshape(-1, 3))
        d = _abi.SurfaceMeshDesc()
        self._lib.cn_surface_mesh_desc_defaults(C.byref(d))
        d.owner_kind = {"soft_body": 0, "cloth": 1}[owner]
        d.owner_index = index
        d.vertex_count = pos.shape[0]
        d.positions = _f32(pos)
        d.normals = _f32(nrm) if nrm is not None else None
        d.index_count = idx.size
        d.indices = _u32(idx) if idx.size else None
        d.match_epsilon = match_epsilon
        out = C.c_uint32()
        _check(self._lib.cn_world_add_surface_mesh(self._h, C.byref(d), C.byref(out)))
        return out.value

    def set_surface_render(self, bindings, fallback_normals, triangle_ranges, triangle_indices, triangles,
                           surface_ranges) -> None:
        """PhysicsWorld::setSurfaceDeformableRenderData with caller-built arrays: bindings (V, 8)
        (4 particle indices as uint32 bits, 4 weights), fallback normals (V, 4), per-vertex
        (start, count) ranges (V, 2) into triangle_indices, triangles (T, 3) particle indices,
        surface particle ranges (S, 2).  None restores the meshes added with add_surface_mesh."""
        if bindings is None:
            _check(self._lib.cn_world_set_surface_render(self._h, None))
            return
        b = np.ascontiguousarray(np.asarray(bindings).view(np.uint32).reshape(-1, 8))
        fn = np.ascontiguousarray(np.asarray(fallback_normals, dtype=np.float32).reshape(-1, 4))
        rg = np.zeros((b.shape[0], 4), np.uint32)
        rg[:, :2] = np.asarray(triangle_ranges, dtype=np.uint32).reshape(-1, 2)
        ti = np.ascontiguousarray(np.asarray(triangle_indices, dtype=np.uint32).reshape(-1))
        tr = np.zeros((np.asarray(triangles).reshape(-1, 3).shape[0], 4), np.uint32)
        tr[:, :3] = np.asarray(triangles, dtype=np.uint32).reshape(-1, 3)
        sr = np.ascontiguousarray(np.asarray(surface_ranges, dtype=np.uint32).reshape(-1, 2))
        d = _abi.SurfaceRenderData()
        d.vertex_count = b.shape[0]
        d.vertex_bindings = C.cast(b.ctypes.data, C.POINTER(_abi.SurfaceVertexBinding))
        d.fallback_normals = _f32(fn)
        d.vertex_triangle_ranges = C.cast(rg.ctypes.data, C.POINTER(_abi.SurfaceTriangleRange))
        d.vertex_triangle_index_count = ti.size
        d.vertex_triangle_indices = _u32(ti) if ti.size else None
        d.triangle_count = tr.shape[0]
        d.triangle_particle_indices = _u32(tr) if tr.size else None
        d.surface_count = sr.shape[0]
        d.surface_particle_ranges = _u32(sr) if sr.size else None
        _check(self._lib.cn_world_set_surface_render(self._h, C.byref(d)))

    def soa(self) -> _abi.WorldSoA:
        s = _abi.WorldSoA()
        _check(self._lib.cn_world_get_soa(self._h, C.byref(s)))
        self._soa = s
        return s

    # views into the packed SoA (valid until the next add_* call)
    def positions(self) -> np.ndarray:
        s = self._soa or self.soa()
        return _view(s.positions_inv_mass, s.particle_count, np.float32, 4)

    def velocities(self) -> np.ndarray:
        s = self._soa or self.soa()
        return _view(s.velocities, s.particle_count, np.float32, 4)

    def layout_mapping(self) -> dict:
        """ParticleLayoutMapping (include/engine/particle_layout_mapping.h): per-particle arrays and
        per-owner (ids, environment, particle offset, particle count), as numpy copies."""
        m = _abi.ParticleLayoutMapping()
        _check(self._lib.cn_world_particle_layout_mapping(self._h, C.byref(m)))
        n = m.particle_count
        out = {"particle_count": n, "soft_body_count": m.soft_body_count, "cloth_count": m.cloth_count,
               "fluid_count": m.fluid_count, "strand_count": m.strand_count,
               "layout_revision": m.layout_revision}
        for name in ("environment_indices", "particle_kinds", "owner_types", "owner_indices", "strand_ids",
                     "strand_orders", "strand_roles", "owning_soft_body_indices", "particle_material_indices",
                     "fluid_material_indices", "phases", "collision_layers", "collision_masks",
                     "adjacency_offsets", "adjacency_counts"):
            out[name] = _view(getattr(m, name), n, np.uint32).copy()
        for owner in ("soft_bodies", "cloths", "fluids", "strands"):
            r = getattr(m, owner)
            ids = np.ctypeslib.as_array(r.ids, (r.count,)).copy() if r.count else np.zeros(0, np.uint64)
            out[owner] = {"ids": ids,
                          "environment_indices": _view(r.environment_indices, r.count, np.uint32).copy(),
                          "particle_offsets": _view(r.particle_offsets, r.count, np.uint32).copy(),
                          "particle_counts": _view(r.particle_counts, r.count, np.uint32).copy()}
        return out

    def counts(self) -> dict:
        s = self._soa or self.soa()
        return {"particles": s.particle_count, "edges": s.edge_count, "bends": s.bend_count,
                "dihedrals": s.dihedral_count, "tets": s.tet_count, "segments": s.strand_segment_count,
                "joints": s.strand_joint_count, "distances": s.strand_distance_count,
                "bodies": s.rigid_body_count, "colliders": s.collider_count,
                "fluid_materials": s.fluid_material_count}

    def fluid_materials(self) -> np.ndarray:
        s = self._soa or self.soa()
        return _view(s.fluid_materials, s.fluid_material_count, np.float32, 12)

    def array(self, name: str) -> np.ndarray:
        """Raw view of one SoA array, e.g. ``array("kinds")`` or ``array("tets")``."""
        s = self._soa or self.soa()
        n = s.particle_count
        spec = {"kinds": ("kinds", n, np.uint32, 1), "metadata": ("metadata", n, np.uint32, 4),
                "radii": ("radii", n, np.float32, 1),
                "tets": ("tets", s.tet_count, np.uint32, 8), "edges": ("edges", s.edge_count, np.uint32, 8),
                "dihedrals": ("dihedrals", s.dihedral_count, np.uint32, 8),
                "segments": ("strand_segments", s.strand_segment_count, np.uint32, 8),
                "joints": ("strand_joints", s.strand_joint_count, np.uint32, 8),
                "body_inverse_inertia": ("body_inverse_inertia", s.rigid_body_count, np.float32, 4),
                "body_types": ("body_types", s.rigid_body_count, np.uint32, 1)}[name]
        return _view(getattr(s, spec[0]), spec[1], spec[2], spec[3])


class Solver:
    """PhysicsSolver mirror (include/physics/physics_solver.h:150-205) on one CUDA device."""

    def __init__(self, desc: Optional[_abi.SolverDesc] = None, device: int = 0):
        self._lib = load()
        self.desc = desc if desc is not None else solver_desc()
        h = C.c_void_p()
        _check(self._lib.cn_solver_create(C.byref(self.desc), device, C.byref(h)))
        self._h = h
        self._n = 0
        self._world = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cn_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync_world(self, world: "World | _abi.WorldSoA") -> None:
        soa = world.soa() if isinstance(world, World) else world
        if isinstance(world, World):
            self._world = world
        _check(self._lib.cn_solver_sync_world(self._h, C.byref(soa)))
        self._n = soa.particle_count
        self._segments = soa.strand_segment_count
        self._bodies = soa.rigid_body_count

    def step(self, dt: float, stream: int = 0) -> None:
        _check(self._lib.cn_solver_step(self._h, dt, C.c_void_p(stream) if stream else None))

    def step_many(self, dt: float, steps: int, stream: int = 0) -> None:
        _check(self._lib.cn_solver_step_many(self._h, dt, steps, C.c_void_p(stream) if stream else None))

    def validate_gpu_meta(self) -> dict:
        m = _abi.Meta()
        status = self._lib.cn_solver_validate_meta(self._h, C.byref(m))
        out = {name: getattr(m, name) for name, _ in _abi.Meta._fields_ if name != "reserved"}
        out["status"] = STATUS.get(status, status)
        return out

    def set_gravity(self, g) -> None:
        _check(self._lib.cn_solver_set_gravity(self._h, *map(float, g)))

    def set_kinematic_target(self, body: int, position, orientation=(0, 0, 0, 1)) -> None:
        p = (C.c_float * 3)(*position)
        q = (C.c_float * 4)(*orientation)
        _check(self._lib.cn_solver_set_kinematic_target(self._h, body, p, q))

    def set_debug(self, keep_fluid_delta=False, post_update_neighbors=False, force_broadphase=False,
                  walk_cells=False) -> None:
        flags = ((1 if keep_fluid_delta else 0) | (2 if post_update_neighbors else 0) | (4 if force_broadphase else 0)
                 | (8 if walk_cells else 0))
        _check(self._lib.cn_solver_set_debug(self._h, flags))

    def set_timing(self, enable: bool = True) -> None:
        _check(self._lib.cn_solver_set_timing(self._h, int(enable)))

    def kernel_times(self) -> dict:
        n = C.c_uint32()
        _check(self._lib.cn_solver_kernel_times(self._h, None, 0, C.byref(n)))
        arr = (_abi.KernelTime * max(n.value, 1))()
        _check(self._lib.cn_solver_kernel_times(self._h, arr, n.value, C.byref(n)))
        return {arr[i].name.decode(): (arr[i].milliseconds, arr[i].launches) for i in range(n.value)}

    def read_rigid_bodies(self, count: Optional[int] = None):
        """(positions with inverse mass, orientations, linear, angular velocities), each (B, 4)."""
        n = self._bodies if count is None else count
        out = [np.zeros((n, 4), np.float32) for _ in range(4)]
        _check(self._lib.cn_solver_read_rigid_bodies(self._h, *(a.ctypes.data for a in out), n))
        return tuple(out)

    def read_surface_render(self):
        """(render positions V x 4, render normals V x 4, surface world AABBs S x 8) after the last frame."""
        v = _abi.SurfaceRenderView()
        _check(self._lib.cn_solver_surface_render_view(self._h, C.byref(v)))
        pos = np.zeros((v.vertex_count, 4), np.float32)
        nrm = np.zeros((v.vertex_count, 4), np.float32)
        box = np.zeros((v.surface_count, 8), np.float32)
        _check(self._lib.cn_solver_read_surface_render(self._h, pos.ctypes.data, nrm.ctypes.data, box.ctypes.data))
        return pos, nrm, box

    def surface_render_view(self) -> dict:
        v = _abi.SurfaceRenderView()
        _check(self._lib.cn_solver_surface_render_view(self._h, C.byref(v)))
        return {name: getattr(v, name) for name, _ in _abi.SurfaceRenderView._fields_}

    def graph_stats(self) -> tuple:
        k, t = C.c_uint32(), C.c_uint32()
        _check(self._lib.cn_solver_graph_stats(self._h, C.byref(k), C.byref(t)))
        return k.value, t.value

    def schedule_info(self) -> dict:
        """The XPBD schedule in use: xpbd_schedule, fused_iterations (1: one cluster kernel per
        substep), cluster_ctas, threads_per_cta, colours per family (edges, strand segments,
        bends + dihedrals, strand joints, strand distances, tets), branches (iteration work on
        side streams: 1 fluid chain, 2 strand families, 4 cloth bends)."""
        v = _abi.ScheduleInfo()
        _check(self._lib.cn_solver_schedule_info(self._h, C.byref(v)))
        out = {name: getattr(v, name) for name, _ in _abi.ScheduleInfo._fields_}
        out["colours"] = dict(zip(("edges", "segments", "bends", "joints", "distances", "tets"), v.colours))
        return out

    def gpu_scene_view(self) -> dict:
        v = _abi.SceneView()
        _check(self._lib.cn_solver_scene_view(self._h, C.byref(v)))
        return {name: getattr(v, name) for name, _ in _abi.SceneView._fields_ if name != "reserved"}

    def export_dlpack(self, buffer: str = "positions_inv_mass"):
        """A torch tensor viewing one device buffer of the scene (no copy; the reference's
        shared_buffer_to_dlpack).  Valid while gpu_scene_view()["binding_generation"] is unchanged."""
        import torch
        ptr = C.c_void_p()
        _check(self._lib.cn_solver_export_dlpack(self._h, buffer.encode(), C.byref(ptr)))
        new_capsule = C.pythonapi.PyCapsule_New
        new_capsule.restype = C.py_object
        new_capsule.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p]
        return torch.utils.dlpack.from_dlpack(new_capsule(ptr, b"dltensor", None))

    SYNC = {"particle_state": 1, "particle_attributes": 2, "constraints": 4, "rigid_bodies": 8, "colliders": 16,
            "surface_render": 32}

    def update_world(self, world: "World | _abi.WorldSoA", *categories: str) -> None:
        """Uploads the named categories (SYNC keys; all when none is named) into the existing
        buffers: the element counts must be the synced ones."""
        soa = world.soa() if isinstance(world, World) else world
        flags = 0
        for c in categories or tuple(self.SYNC):
            flags |= self.SYNC[c]
        _check(self._lib.cn_solver_update_world(self._h, C.byref(soa), flags))

    def read_particles(self):
        x = np.zeros((self._n, 4), np.float32)
        v = np.zeros((self._n, 4), np.float32)
        xp = np.zeros((self._n, 4), np.float32)
        _check(self._lib.cn_solver_read_particles(self._h, _f32(x), _f32(v), _f32(xp), self._n))
        return x, v, xp

    def write_particles(self, x: Optional[np.ndarray] = None, v: Optional[np.ndarray] = None) -> None:
        xa = np.ascontiguousarray(x, dtype=np.float32) if x is not None else None
        va = np.ascontiguousarray(v, dtype=np.float32) if v is not None else None
        _check(self._lib.cn_solver_write_particles(self._h, _f32(xa) if xa is not None else None,
                                                   _f32(va) if va is not None else None, self._n))

    def read_strand_orientations(self) -> np.ndarray:
        q = np.zeros((self._segments, 4), np.float32)
        if self._segments:
            _check(self._lib.cn_solver_read_strand_orientations(self._h, _f32(q), self._segments))
        return q

    def debug_read(self, name: str) -> np.ndarray:
        which = DEBUG[name]
        size = C.c_size_t()
        _check(self._lib.cn_solver_debug_read(self._h, which, None, 0, C.byref(size)))
        buf = np.zeros(size.value, np.uint8)
        _check(self._lib.cn_solver_debug_read(self._h, which, buf.ctypes.data_as(C.c_void_p), size.value,
                                              C.byref(size)))
        return buf


def batch_desc(solver: Optional[_abi.SolverDesc] = None, **fields) -> _abi.BatchDesc:
    """cn_batch_desc with defaults, the shared solver settings and field overrides."""
    d = _abi.BatchDesc()
    load().cn_batch_desc_defaults(C.byref(d))
    if solver is not None:
        d.solver = solver
    for key, value in fields.items():
        setattr(d, key, value)
    return d


def _stream(stream) -> Optional[C.c_void_p]:
    return C.c_void_p(stream) if stream else None


class Batch:
    """Independent soft-tissue scenes resident in one device pool, stepped together (cn_batch_*)."""

    def __init__(self, desc: Optional[_abi.BatchDesc] = None, device: int = 0):
        self._lib = load()
        self.desc = desc if desc is not None else batch_desc()
        h = C.c_void_p()
        _check(self._lib.cn_batch_create(C.byref(self.desc), device, C.byref(h)))
        self._h = h
        self._sizes = {}
        self._servers = weakref.WeakSet()   # servers over this batch, closed before it

    def close(self):
        if getattr(self, "_h", None):
            for srv in list(getattr(self, "_servers", ())):
                srv.close()
            self._lib.cn_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_scene(self, world: "World | _abi.WorldSoA") -> int:
        soa = world.soa() if isinstance(world, World) else world
        out = C.c_uint32()
        _check(self._lib.cn_batch_add_scene(self._h, C.byref(soa), C.byref(out)))
        self._sizes[out.value] = soa.particle_count
        return out.value

    def remove_scene(self, scene: int) -> None:
        _check(self._lib.cn_batch_remove_scene(self._h, scene))
        self._sizes.pop(scene, None)

    def set_kinematic_target(self, scene: int, body: int, position, orientation=(0, 0, 0, 1)) -> None:
        p = (C.c_float * 3)(*position)
        q = (C.c_float * 4)(*orientation)
        _check(self._lib.cn_batch_set_kinematic_target(self._h, scene, body, p, q))

    def step(self, scenes: Sequence[int], dt: float, stream: int = 0) -> None:
        ids = np.ascontiguousarray(np.asarray(scenes, dtype=np.uint32))
        _check(self._lib.cn_batch_step(self._h, _u32(ids), ids.size, dt, _stream(stream)))

    def read_particles(self, scene: int):
        n = self._sizes[scene]
        x = np.zeros((n, 4), np.float32)
        v = np.zeros((n, 4), np.float32)
        _check(self._lib.cn_batch_read_particles(self._h, scene, _f32(x), _f32(v), n))
        return x, v

    def stats(self) -> dict:
        s = _abi.BatchStats()
        _check(self._lib.cn_batch_get_stats(self._h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in _abi.BatchStats._fields_ if not name.startswith("reserved")}

    def set_schedule(self, tile_elements: int, blocks_per_sm: int) -> None:
        _check(self._lib.cn_batch_set_schedule(self._h, tile_elements, blocks_per_sm))

    def set_fused(self, cluster_ctas: int) -> None:
        """0: per-phase iteration kernels; 1, 2, 4 or 8: the persistent fused iterations, one
        cluster of that many CTAs per scene at a time."""
        _check(self._lib.cn_batch_set_fused(self._h, cluster_ctas))

    def set_xpbd_schedule(self, schedule: int) -> None:
        """XPBD_GATHER, or (in a batch created with a coloured schedule) XPBD_COLOUR_JACOBI /
        XPBD_COLOUR_GAUSS_SEIDEL for the next ticks."""
        _check(self._lib.cn_batch_set_xpbd_schedule(self._h, schedule))

    def autotune(self, scenes: Sequence[int], dt: float) -> dict:
        ids = np.ascontiguousarray(np.asarray(scenes, dtype=np.uint32))
        t = _abi.BatchTuning()
        _check(self._lib.cn_batch_autotune(self._h, _u32(ids), ids.size, dt, C.byref(t)))
        return {"tile_elements": t.tile_elements, "blocks_per_sm": t.blocks_per_sm, "tick_ms": t.tick_ms,
                "cluster_ctas": t.cluster_ctas, "xpbd_schedule": t.xpbd_schedule,
                "candidates": [(t.candidates[k].tile_elements, t.candidates[k].blocks_per_sm,
                                round(t.candidates[k].tick_ms, 4), t.candidates[k].cluster_ctas,
                                t.candidates[k].xpbd_schedule)
                               for k in range(t.candidate_count)]}


class Server:
    """Serving loop over a Batch (cn_server_*): registration, admission by the memory budget,
    continuous batching of pending requests, per-request latency."""

    def __init__(self, batch: Batch, frame_dt: float, max_scenes_per_tick: int = 0):
        self._lib = load()
        self.batch = batch
        d = _abi.ServerDesc()
        self._lib.cn_server_desc_defaults(C.byref(d))
        d.frame_dt = frame_dt
        d.max_scenes_per_tick = max_scenes_per_tick
        h = C.c_void_p()
        _check(self._lib.cn_server_create(batch._h, C.byref(d), batch.desc.solver.substeps, C.byref(h)))
        self._h = h
        self._sizes = []
        batch._servers.add(self)

    def close(self):
        # a server is destroyed before its batch (the batch's close() closes it first)
        if getattr(self, "_h", None):
            if getattr(self.batch, "_h", None):
                self._lib.cn_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def register(self, world: "World | _abi.WorldSoA") -> int:
        soa = world.soa() if isinstance(world, World) else world
        out = C.c_uint32()
        _check(self._lib.cn_server_register_scene(self._h, C.byref(soa), C.byref(out)))
        self._sizes.append(soa.particle_count)
        return out.value

    def admit(self, scene: int) -> bool:
        """Makes a scene resident ahead of its requests; False when the budget has no room."""
        st = self._lib.cn_server_admit(self._h, scene)
        if st == 5:  # CN_ERR_CAPACITY
            return False
        _check(st)
        return True

    def submit(self, scene: int, steps: int, tool_body: int = 0, targets=None) -> int:
        rid = C.c_uint64()
        tp = None
        if targets is not None:
            arr = np.ascontiguousarray(np.asarray(targets, dtype=np.float32).reshape(steps, 7))
            tp = _f32(arr)
        _check(self._lib.cn_server_submit(self._h, scene, steps, tool_body, tp, C.byref(rid)))
        return rid.value

    def tick(self, stream: int = 0) -> int:
        n = C.c_uint32()
        _check(self._lib.cn_server_tick(self._h, _stream(stream), C.byref(n)))
        return n.value

    def drain(self, stream: int = 0) -> None:
        _check(self._lib.cn_server_drain(self._h, _stream(stream)))

    def poll(self) -> list:
        out = (_abi.RequestDone * 4096)()
        got, n = [], C.c_uint32()
        while True:
            _check(self._lib.cn_server_poll(self._h, out, 4096, C.byref(n)))
            got += [{"request": out[k].request_id, "scene": out[k].scene, "steps": out[k].steps,
                     "submit_s": out[k].submit_s, "first_tick_s": out[k].first_tick_s, "done_s": out[k].done_s}
                    for k in range(n.value)]
            if n.value < 4096:
                return got

    def stats(self) -> dict:
        s = _abi.ServerStats()
        _check(self._lib.cn_server_get_stats(self._h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in _abi.ServerStats._fields_}

    def read_particles(self, scene: int):
        n = self._sizes[scene]
        x = np.zeros((n, 4), np.float32)
        v = np.zeros((n, 4), np.float32)
        _check(self._lib.cn_server_read_particles(self._h, scene, _f32(x), _f32(v), n))
        return x, v
