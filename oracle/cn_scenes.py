"""TEST INFRASTRUCTURE ONLY: the PBF dam break built for the oracle without the product library.

bench.py's reference arm times the oracle (the CPU restatement of the reference's substep) on the
benchmark scene.  So that the arm never loads libcn_physics.so, this module restates the
scene authoring the dam break needs, in numpy, from the reference's PhysicsWorld:

  * the fluid lattice of a FluidState with a RegularGrid source (src/physics/physics_world.cpp:
    6857-6891): round(size / spacing) points per axis, cell centres at
    -size / 2 + (i + 0.5) * spacing, moved by the rest transform (identity rotation and scale);
  * the fluid solver material (physics_world.cpp:97-262), taken from the oracle's own
    restatement (cno_fluid_material);
  * the particle SoA packing of a lone fluid (physics_world.cpp:4919-5400): inverse mass 1/mass,
    kind Fluid, metadata (environment, phase = group | self-collide, layer, mask), owner Fluid;
  * the grid cell size max(2 r, h) (physics_world.cpp:6829-6846);
  * one static body with five box colliders (the walls and floor of the benchmark box);
  * the solver defaults of PhysicsSolverDesc (include/physics/physics_solver.h:22-143).

tests/test_oracle_scenes.py checks that the arrays are byte-identical to the product's World
for the same arguments.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import cn_oracle

PHASE_SELF_COLLIDE = 0x80000000
OWNER_FLUID = 2
KIND_FLUID = 1
SHAPE_BOX = 1


def _abi():
    # The C ABI's struct layouts (plain ctypes; importing them loads no library).
    from cn_physics import _abi as abi
    return abi


def reference_desc(**overrides):
    """PhysicsSolverDesc defaults (physics_solver.h:22-143) in the C ABI's cn_solver_desc."""
    abi = _abi()
    d = abi.SolverDesc()
    d.gravity = (C.c_float * 3)(0.0, -9.81, 0.0)
    d.substeps = 1
    d.default_iterations = 20
    for name, vals in (("contact", (1.0e-3, 4.0, 0.95, 0.05, 0.5, 2.0, 0.0, 1.0e-5)),
                       ("rigid", (0.25, 0.90, 0.10, 1.0, 0.01, 0.10, 0.8, 0.5)),
                       ("joints", (0.95, 0.7, 0.05, 0.02, 0.12, 1.0e-5, 5.0e-5, 1.0e-5))):
        part = getattr(d, name)
        for field, v in zip(part._fields_, vals):
            setattr(part, field[0], v)
    d.soft.internal_relaxation = 0.2
    d.fluid.constraint_relaxation = 0.7
    d.fluid.position_relaxation = 1.0
    d.fluid.boundary_density_scale = 0.12
    d.fluid.boundary_delta_scale = 0.08
    d.fluid.max_under_density_ratio = 0.0
    d.enable_blocking_readback = 1
    d.max_fluid_neighborhood = 128
    d.particle_rigid_pairs_per_particle = 8
    for k, v in overrides.items():
        setattr(d, k, v)
    return d


class DamBreak:
    """A fluid block in a box of static walls, as a cn_world_soa over numpy arrays (kept alive
    by this object).  Arguments and defaults are those of the benchmark scene."""

    def __init__(self, nx=128, ny=64, nz=128, spacing=0.05, seed=0, box=(12.8, 6.4, 25.6)):
        f = np.float32
        # scene arguments are formed in double precision and handed over as float32 (as the
        # benchmark's scene builder passes them through the C ABI's descriptors)
        r = 0.6 * spacing
        size_d = (nx * spacing, ny * spacing, nz * spacing)
        offset = r - 0.5 * spacing
        center = tuple(f(s * 0.5 + offset) for s in size_d)
        size = tuple(f(s) for s in size_d)
        sp = f(spacing)
        r = f(r)
        counts = [max(1, int(np.floor(s / sp + f(0.5)))) for s in size]
        axes = [(-s * f(0.5)) + (np.arange(n, dtype=f) + f(0.5)) * sp for s, n in zip(size, counts)]
        # rest transform: scale 1 and identity rotation leave the lattice point as it is (a
        # rotation by (0, 0, 0, 1) adds exact zeros), then the translation
        z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
        n = x.size
        pos = np.empty((n, 4), f)
        pos[:, 0] = (x.ravel() + f(0.0)) + center[0]
        pos[:, 1] = (y.ravel() + f(0.0)) + center[1]
        pos[:, 2] = (z.ravel() + f(0.0)) + center[2]
        pos[:, 3] = f(1.0)
        rng = np.random.default_rng(seed)
        jitter = rng.uniform(-1.0e-4, 1.0e-4, size=(n, 3)).astype(f)
        pos[:, :3] += jitter
        self.positions = pos
        self.velocities = np.zeros((n, 4), f)
        self.radii = np.full(n, r, f)
        self.kinds = np.full(n, KIND_FLUID, np.uint32)
        meta = np.zeros((n, 4), np.uint32)
        meta[:, 1] = PHASE_SELF_COLLIDE
        meta[:, 2] = 1
        meta[:, 3] = 0xFFFFFFFF
        self.metadata = meta
        self.material_indices = np.zeros(n, np.uint32)
        self.fluid_material_indices = np.zeros(n, np.uint32)
        self.owner_types = np.full(n, OWNER_FLUID, np.uint32)
        self.owner_indices = np.zeros(n, np.uint32)
        self.adjacency_offsets = np.zeros(n, np.uint32)
        self.adjacency_counts = np.zeros(n, np.uint32)
        self.contact_materials = np.zeros((1, 4), f)   # normalised default: no friction
        self.fluid_materials = cn_oracle.fluid_material(float(r), viscosity=0.01).reshape(1, 12)
        # cn_fluid_material / GpuFluidMaterial: smoothing radius is the third field
        self.cell_size = f(max(float(f(2.0) * r), float(self.fluid_materials[0, 2]), 1.0e-4))
        # one static body, five box colliders (floor, x walls, z walls)
        bx, by, bz = box
        t = 0.5
        boxes = [((bx * 0.5 + 2 * t, t, bz * 0.5 + 2 * t), (bx * 0.5, -t, bz * 0.5)),
                 ((t, by * 0.5 + 2 * t, bz * 0.5 + 2 * t), (-t, by * 0.5, bz * 0.5)),
                 ((t, by * 0.5 + 2 * t, bz * 0.5 + 2 * t), (bx + t, by * 0.5, bz * 0.5)),
                 ((bx * 0.5 + 2 * t, by * 0.5 + 2 * t, t), (bx * 0.5, by * 0.5, -t)),
                 ((bx * 0.5 + 2 * t, by * 0.5 + 2 * t, t), (bx * 0.5, by * 0.5, bz + t))]
        geo = np.zeros((5, 12), f)
        bp = np.zeros((5, 8), np.uint32)
        for c, (half, local) in enumerate(boxes):
            geo[c, 0:3] = half
            geo[c, 4:7] = local
            geo[c, 8:12] = (0.0, 0.0, 0.0, 1.0)
            bp[c] = (0, SHAPE_BOX, 0, 1, 0xFFFFFFFF, 1, 0, 0)
        self.collider_geometry = geo
        self.collider_broadphase = bp
        self.collider_materials = np.tile(np.array([0.5, 0.0, 0.0, 0.5], f), (5, 1))
        self.body_positions = np.zeros((1, 4), f)
        self.body_orientations = np.array([[0, 0, 0, 1]], f)
        self.body_zero = np.zeros((1, 4), f)
        self.body_scales = np.array([[1, 1, 1, 0]], f)
        self.body_types = np.zeros(1, np.uint32)
        self.body_kin_flags = np.zeros(1, np.uint32)
        self.body_collider_ranges = np.array([[0, 5]], np.uint32)
        self.body_collider_indices = np.arange(5, dtype=np.uint32)
        self.desc = reference_desc(substeps=2, fluid_iterations=4, enable_blocking_readback=0)
        self.frame_dt = 1.0 / 120.0
        self._soa = self._pack()

    def _pack(self):
        abi = _abi()
        s = abi.WorldSoA()
        fp = lambda a: a.ctypes.data_as(abi.P_f32)
        up = lambda a: a.ctypes.data_as(abi.P_u32)
        s.particle_count = self.positions.shape[0]
        s.positions_inv_mass = fp(self.positions)
        s.velocities = fp(self.velocities)
        s.radii = fp(self.radii)
        s.kinds = up(self.kinds)
        s.metadata = up(self.metadata)
        s.material_indices = up(self.material_indices)
        s.fluid_material_indices = up(self.fluid_material_indices)
        s.owner_types = up(self.owner_types)
        s.owner_indices = up(self.owner_indices)
        s.adjacency_offsets = up(self.adjacency_offsets)
        s.adjacency_counts = up(self.adjacency_counts)
        s.adjacency_index_count = 0
        s.particle_grid_cell_size = float(self.cell_size)
        s.contact_material_count = 1
        s.contact_materials = fp(self.contact_materials)
        s.fluid_material_count = 1
        s.fluid_materials = self.fluid_materials.ctypes.data
        s.rigid_body_count = 1
        s.body_positions_inv_mass = fp(self.body_positions)
        s.body_orientations = fp(self.body_orientations)
        s.body_linear_velocities = fp(self.body_zero)
        s.body_angular_velocities = fp(self.body_zero)
        s.body_scales = fp(self.body_scales)
        s.body_inverse_inertia = fp(self.body_zero)
        s.body_types = up(self.body_types)
        s.body_kinematic_target_positions = fp(self.body_zero)
        s.body_kinematic_target_orientations = fp(self.body_orientations)
        s.body_kinematic_target_flags = up(self.body_kin_flags)
        s.body_collider_ranges = up(self.body_collider_ranges)
        s.body_collider_indices = up(self.body_collider_indices)
        s.body_collider_index_count = 5
        s.collider_count = 5
        s.collider_geometry = self.collider_geometry.ctypes.data
        s.collider_broadphase = self.collider_broadphase.ctypes.data
        s.collider_materials = fp(self.collider_materials)
        return s

    def soa(self):
        return self._soa
