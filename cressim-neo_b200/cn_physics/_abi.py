"""ctypes mirror of include/cn_physics.h (the C ABI of the particle substep library)."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent.parent / "libcn_physics.so"

u32 = C.c_uint32
f32 = C.c_float
P_f32 = C.POINTER(C.c_float)
P_u32 = C.POINTER(C.c_uint32)


class ContactSettings(C.Structure):
    _fields_ = [(n, f32) for n in (
        "slop", "manifold_merge_slop_multiplier", "soft_relaxation", "soft_max_correction_per_iteration",
        "restitution_velocity_threshold", "restitution_penetration_slop_multiplier",
        "rigid_restitution_velocity_threshold", "position_friction_min_distance")]


class RigidSettings(C.Structure):
    _fields_ = [(f"f{i}", f32) for i in range(8)]


class JointSettings(C.Structure):
    _fields_ = [(f"f{i}", f32) for i in range(8)]


XPBD_GATHER, XPBD_COLOUR_JACOBI, XPBD_COLOUR_GAUSS_SEIDEL = 0, 1, 2
FUSED_OFF, FUSED_ON = 0, 1


class SoftSettings(C.Structure):
    _fields_ = [("internal_relaxation", f32), ("xpbd_schedule", u32), ("fused_iterations", u32),
                ("reserved", f32 * 5)]


class ScheduleInfo(C.Structure):
    _fields_ = [("xpbd_schedule", u32), ("fused_iterations", u32), ("cluster_ctas", u32),
                ("threads_per_cta", u32), ("colours", u32 * 6), ("branches", u32)]


class FluidSettings(C.Structure):
    _fields_ = [("constraint_relaxation", f32), ("position_relaxation", f32),
                ("boundary_density_scale", f32), ("boundary_delta_scale", f32),
                ("max_under_density_ratio", f32), ("reserved", f32 * 3)]


class SolverDesc(C.Structure):
    _fields_ = [("gravity", f32 * 3), ("substeps", u32), ("default_iterations", u32),
                ("fluid_iterations", u32), ("soft_internal_iterations", u32),
                ("soft_contact_iterations", u32), ("rigid_joint_iterations", u32),
                ("rigid_rigid_contact_iterations", u32), ("contact", ContactSettings),
                ("rigid", RigidSettings), ("joints", JointSettings), ("soft", SoftSettings),
                ("fluid", FluidSettings), ("enable_blocking_readback", u32),
                ("max_fluid_neighborhood", u32), ("particle_rigid_pairs_per_particle", u32)]


class FluidMaterial(C.Structure):
    _fields_ = [(n, f32) for n in (
        "rest_density", "inv_rest_density", "smoothing_radius", "density_constraint_scale",
        "viscosity", "cohesion", "cohesion1", "cohesion2", "surface_tension",
        "vorticity_confinement", "gravity_scale", "cfl_radius")]


class SurfaceVertexBinding(C.Structure):
    _fields_ = [("particle_indices", u32 * 4), ("weights", f32 * 4)]


class SurfaceTriangleRange(C.Structure):
    _fields_ = [("start", u32), ("count", u32), ("reserved0", u32), ("reserved1", u32)]


class SurfaceRenderData(C.Structure):
    _fields_ = [
        ("vertex_count", u32), ("vertex_bindings", C.POINTER(SurfaceVertexBinding)), ("fallback_normals", P_f32),
        ("vertex_triangle_ranges", C.POINTER(SurfaceTriangleRange)), ("vertex_triangle_index_count", u32),
        ("vertex_triangle_indices", P_u32), ("triangle_count", u32), ("triangle_particle_indices", P_u32),
        ("surface_count", u32), ("surface_particle_ranges", P_u32)]


class SurfaceMeshDesc(C.Structure):
    _fields_ = [("owner_kind", u32), ("owner_index", u32), ("vertex_count", u32), ("positions", P_f32),
                ("normals", P_f32), ("index_count", u32), ("indices", P_u32), ("match_epsilon", f32),
                ("reserved", u32 * 3)]


class SurfaceRenderView(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("render_positions", "render_normals", "triangle_normals", "chunk_aabbs",
                                           "world_aabbs")] + [
        (n, u32) for n in ("vertex_count", "triangle_count", "chunk_count", "surface_count")] + [
        ("binding_generation", C.c_uint64)]


class WorldSoA(C.Structure):
    _fields_ = [
        ("particle_count", u32), ("positions_inv_mass", P_f32), ("velocities", P_f32), ("radii", P_f32),
        ("kinds", P_u32), ("metadata", P_u32), ("material_indices", P_u32), ("fluid_material_indices", P_u32),
        ("owner_types", P_u32), ("owner_indices", P_u32), ("adjacency_offsets", P_u32),
        ("adjacency_counts", P_u32), ("adjacency_indices", P_u32), ("adjacency_index_count", u32),
        ("particle_grid_cell_size", f32),
        ("contact_material_count", u32), ("contact_materials", P_f32),
        ("fluid_material_count", u32), ("fluid_materials", C.c_void_p),
        ("edge_count", u32), ("edges", C.c_void_p),
        ("bend_count", u32), ("bends", C.c_void_p),
        ("dihedral_count", u32), ("dihedrals", C.c_void_p),
        ("tet_count", u32), ("tets", C.c_void_p),
        ("strand_segment_count", u32), ("strand_segments", C.c_void_p),
        ("strand_segment_orientations", P_f32),
        ("strand_joint_count", u32), ("strand_joints", C.c_void_p),
        ("strand_distance_count", u32), ("strand_distances", C.c_void_p),
        ("rigid_body_count", u32), ("body_positions_inv_mass", P_f32), ("body_orientations", P_f32),
        ("body_linear_velocities", P_f32), ("body_angular_velocities", P_f32), ("body_scales", P_f32),
        ("body_inverse_inertia", P_f32), ("body_types", P_u32),
        ("body_kinematic_target_positions", P_f32), ("body_kinematic_target_orientations", P_f32),
        ("body_kinematic_target_flags", P_u32), ("body_collider_ranges", P_u32),
        ("body_collider_indices", P_u32), ("body_collider_index_count", u32),
        ("collider_count", u32), ("collider_geometry", C.c_void_p), ("collider_broadphase", C.c_void_p),
        ("collider_materials", P_f32), ("surface_render", C.POINTER(SurfaceRenderData)),
        ("rigid_proxy_local_positions", P_f32), ("body_proxy_contact_materials", P_f32),
    ]


class OwnerRanges(C.Structure):
    _fields_ = [("count", u32), ("ids", C.POINTER(C.c_uint64)), ("environment_indices", P_u32),
                ("particle_offsets", P_u32), ("particle_counts", P_u32)]


class ParticleLayoutMapping(C.Structure):
    _fields_ = [("particle_count", u32), ("soft_body_count", u32), ("cloth_count", u32), ("fluid_count", u32),
                ("strand_count", u32), ("layout_revision", C.c_uint64)] + \
               [(n, P_u32) for n in ("environment_indices", "particle_kinds", "owner_types", "owner_indices",
                                     "strand_ids", "strand_orders", "strand_roles", "owning_soft_body_indices",
                                     "particle_material_indices", "fluid_material_indices", "phases",
                                     "collision_layers", "collision_masks", "adjacency_offsets",
                                     "adjacency_counts")] + \
               [(n, OwnerRanges) for n in ("soft_bodies", "cloths", "fluids", "strands")]


class Transform(C.Structure):
    _fields_ = [("position", f32 * 3), ("rotation", f32 * 4), ("scale", f32 * 3)]


class ContactMaterialDesc(C.Structure):
    _fields_ = [("friction", f32), ("restitution", f32), ("damping", f32), ("static_friction", f32)]


class SoftBodyGridDesc(C.Structure):
    _fields_ = [("size", f32 * 3), ("target_particle_spacing", f32), ("rest_transform", Transform),
                ("particle_mass", f32), ("particle_radius", f32), ("edge_compliance", f32),
                ("volume_compliance", f32), ("self_collision_enabled", u32), ("environment_index", u32),
                ("collision_layer", u32), ("collision_mask", u32), ("material", ContactMaterialDesc),
                ("static_particle_indices", P_u32), ("static_particle_count", u32)]


class FluidGridDesc(C.Structure):
    _fields_ = [("size", f32 * 3), ("target_particle_spacing", f32), ("rest_transform", Transform),
                ("particle_mass", f32), ("particle_radius", f32), ("viscosity", f32), ("cohesion", f32),
                ("surface_tension", f32), ("vorticity_confinement", f32), ("gravity_scale", f32),
                ("cfl_coefficient", f32), ("environment_index", u32), ("collision_layer", u32),
                ("collision_mask", u32), ("material", ContactMaterialDesc)]


class ClothGridDesc(C.Structure):
    _fields_ = [("resolution", u32 * 2), ("size", f32 * 2), ("rest_transform", Transform),
                ("particle_mass", f32), ("particle_radius", f32), ("structural_compliance", f32),
                ("bend_compliance", f32), ("self_collision_enabled", u32), ("environment_index", u32),
                ("collision_layer", u32), ("collision_mask", u32), ("material", ContactMaterialDesc),
                ("static_particle_indices", P_u32), ("static_particle_count", u32)]


class StrandDesc(C.Structure):
    _fields_ = [("rest_positions", P_f32), ("rest_position_count", u32), ("particle_mass", f32),
                ("particle_radius", f32), ("stretch_shear_compliance", f32), ("bend_compliance", f32),
                ("twist_compliance", f32), ("distance_compliance", f32), ("self_collision_enabled", u32),
                ("environment_index", u32), ("collision_layer", u32), ("collision_mask", u32),
                ("material", ContactMaterialDesc), ("static_particle_indices", P_u32),
                ("static_particle_count", u32)]


class RigidBodyDesc(C.Structure):
    _fields_ = [("body_type", u32), ("position", f32 * 3), ("orientation", f32 * 4), ("scale", f32 * 3),
                ("mass", f32), ("inverse_inertia_local", f32 * 3)]


class ColliderDesc(C.Structure):
    _fields_ = [("body", u32), ("shape_type", u32), ("shape_params", f32 * 4), ("local_position", f32 * 3),
                ("local_orientation", f32 * 4), ("enabled", u32), ("friction", f32),
                ("static_friction", f32), ("restitution", f32), ("environment_index", u32),
                ("collision_layer", u32), ("collision_mask", u32)]


class RigidProxyDesc(C.Structure):
    _fields_ = [("body", u32), ("local_positions", P_f32), ("count", u32), ("radius", f32),
                ("material", ContactMaterialDesc), ("environment_index", u32), ("collision_layer", u32),
                ("collision_mask", u32)]


class Meta(C.Structure):
    _fields_ = [(n, u32) for n in (
        "particle_rigid_candidate_count", "required_particle_rigid_candidate_count",
        "particle_rigid_candidate_overflow", "particle_particle_candidate_count",
        "required_particle_particle_candidate_count", "particle_particle_candidate_overflow",
        "fluid_boundary_candidate_overflow", "active_particle_rigid_contact_count",
        "active_particle_contact_count", "fluid_neighbor_truncations", "device_wait_timeouts",
        "rigid_rigid_candidate_count", "required_rigid_rigid_candidate_count", "rigid_rigid_candidate_overflow",
        "proxy_rigid_contact_count", "required_proxy_rigid_contact_count", "proxy_rigid_contact_overflow")] + [
        ("reserved", u32 * 1)]


class SceneView(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "positions_inv_mass", "previous_positions", "velocities", "radii", "kinds", "edges", "bends",
        "dihedrals", "tets", "strand_segments", "strand_joints", "strand_distances",
        "strand_segment_states")] + [(n, u32) for n in (
            "particle_count", "edge_count", "bend_count", "dihedral_count", "tet_count",
            "strand_segment_count", "strand_joint_count", "strand_distance_count")] + [
        ("binding_generation", C.c_uint64), ("device", C.c_int32), ("reserved", u32)]


class KernelTime(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("milliseconds", f32), ("launches", u32)]


# Exported entry points and their signatures: (name, restype, argtypes).
u64 = C.c_uint64


class BatchDesc(C.Structure):
    _fields_ = [("solver", SolverDesc), ("memory_budget_bytes", u64), ("max_scenes", u32),
                ("particle_capacity", u32), ("edge_capacity", u32), ("tet_capacity", u32),
                ("body_capacity", u32), ("collider_capacity", u32), ("tile_elements", u32),
                ("blocks_per_sm", u32), ("rigid_pairs_per_particle", u32), ("fused_cluster_ctas", u32),
                ("reserved", u32 * 2)]


class BatchStats(C.Structure):
    _fields_ = [("resident_scenes", u32), ("particles_used", u32), ("particle_capacity", u32),
                ("edges_used", u32), ("edge_capacity", u32), ("tets_used", u32), ("tet_capacity", u32),
                ("tile_elements", u32), ("grid_blocks", u32), ("fused_cluster_ctas", u32), ("xpbd_schedule", u32),
                ("reserved0", u32), ("budget_bytes", u64),
                ("budget_used_bytes", u64), ("pool_bytes", u64), ("ticks", u64)]


class BatchCandidate(C.Structure):
    _fields_ = [("tile_elements", u32), ("blocks_per_sm", u32), ("tick_ms", f32), ("cluster_ctas", u32),
                ("xpbd_schedule", u32)]


class BatchTuning(C.Structure):
    _fields_ = [("tile_elements", u32), ("blocks_per_sm", u32), ("tick_ms", f32), ("candidate_count", u32),
                ("candidates", BatchCandidate * 24), ("cluster_ctas", u32), ("xpbd_schedule", u32),
                ("reserved", u32 * 2)]


class ServerDesc(C.Structure):
    _fields_ = [("frame_dt", f32), ("max_scenes_per_tick", u32), ("reserved", u32 * 6)]


class RequestDone(C.Structure):
    _fields_ = [("request_id", u64), ("scene", u32), ("steps", u32), ("submit_s", C.c_double),
                ("first_tick_s", C.c_double), ("done_s", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("ticks", u64), ("scene_steps", u64), ("particle_substeps", u64), ("admissions", u64),
                ("evictions", u64), ("completed", u64), ("pending", u64), ("resident_scenes", u32),
                ("registered_scenes", u32), ("gpu_ms", C.c_double), ("tick_ms_p50", f32), ("tick_ms_p99", f32)]


class DiffDesc(C.Structure):
    _fields_ = [("gravity", f32 * 3), ("substeps", u32), ("iterations", u32), ("substep_dt", f32),
                ("relaxation", f32), ("checkpoint_interval", u32), ("precision", u32), ("reserved", u32 * 4)]


SIGNATURES = [
    ("cn_last_error", C.c_char_p, []),
    ("cn_version", C.c_char_p, []),
    ("cn_solver_desc_defaults", None, [C.POINTER(SolverDesc)]),
    ("cn_soft_body_grid_desc_defaults", None, [C.POINTER(SoftBodyGridDesc)]),
    ("cn_fluid_grid_desc_defaults", None, [C.POINTER(FluidGridDesc)]),
    ("cn_cloth_grid_desc_defaults", None, [C.POINTER(ClothGridDesc)]),
    ("cn_strand_desc_defaults", None, [C.POINTER(StrandDesc)]),
    ("cn_rigid_body_desc_defaults", None, [C.POINTER(RigidBodyDesc)]),
    ("cn_collider_desc_defaults", None, [C.POINTER(ColliderDesc)]),
    ("cn_rigid_proxy_desc_defaults", None, [C.POINTER(RigidProxyDesc)]),
    ("cn_world_create", C.c_int, [C.POINTER(C.c_void_p)]),
    ("cn_world_destroy", None, [C.c_void_p]),
    ("cn_world_add_soft_body_grid", C.c_int, [C.c_void_p, C.POINTER(SoftBodyGridDesc), P_u32]),
    ("cn_world_add_soft_body_tet_mesh", C.c_int, [C.c_void_p, C.POINTER(SoftBodyGridDesc), P_f32, C.c_uint32,
                                                  P_u32, C.c_uint32, P_u32]),
    ("cn_world_add_soft_body_tetgen", C.c_int, [C.c_void_p, C.POINTER(SoftBodyGridDesc), C.c_char_p, C.c_char_p,
                                                P_u32]),
    ("cn_world_add_soft_body_meshfree", C.c_int, [C.c_void_p, C.POINTER(SoftBodyGridDesc), P_f32, C.c_uint32,
                                                  C.c_uint32, P_u32]),
    ("cn_world_add_fluid_grid", C.c_int, [C.c_void_p, C.POINTER(FluidGridDesc), P_u32]),
    ("cn_world_add_cloth_grid", C.c_int, [C.c_void_p, C.POINTER(ClothGridDesc), P_u32]),
    ("cn_world_add_strand", C.c_int, [C.c_void_p, C.POINTER(StrandDesc), P_u32]),
    ("cn_world_add_rigid_body", C.c_int, [C.c_void_p, C.POINTER(RigidBodyDesc), P_u32]),
    ("cn_world_add_collider", C.c_int, [C.c_void_p, C.POINTER(ColliderDesc), P_u32]),
    ("cn_world_set_rigid_proxy_particles", C.c_int, [C.c_void_p, C.POINTER(RigidProxyDesc)]),
    ("cn_world_get_soa", C.c_int, [C.c_void_p, C.POINTER(WorldSoA)]),
    ("cn_solver_create", C.c_int, [C.POINTER(SolverDesc), C.c_int, C.POINTER(C.c_void_p)]),
    ("cn_solver_destroy", None, [C.c_void_p]),
    ("cn_solver_sync_world", C.c_int, [C.c_void_p, C.POINTER(WorldSoA)]),
    ("cn_solver_step", C.c_int, [C.c_void_p, f32, C.c_void_p]),
    ("cn_solver_step_many", C.c_int, [C.c_void_p, f32, u32, C.c_void_p]),
    ("cn_solver_validate_meta", C.c_int, [C.c_void_p, C.POINTER(Meta)]),
    ("cn_solver_set_gravity", C.c_int, [C.c_void_p, f32, f32, f32]),
    ("cn_solver_set_kinematic_target", C.c_int, [C.c_void_p, u32, P_f32, P_f32]),
    ("cn_solver_scene_view", C.c_int, [C.c_void_p, C.POINTER(SceneView)]),
    ("cn_solver_surface_render_view", C.c_int, [C.c_void_p, C.POINTER(SurfaceRenderView)]),
    ("cn_solver_read_rigid_bodies", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, u32]),
    ("cn_solver_step_io", C.c_int, [C.c_void_p, f32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("cn_solver_read_surface_render", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("cn_surface_mesh_desc_defaults", None, [C.POINTER(SurfaceMeshDesc)]),
    ("cn_world_add_surface_mesh", C.c_int, [C.c_void_p, C.POINTER(SurfaceMeshDesc), C.POINTER(u32)]),
    ("cn_world_set_surface_render", C.c_int, [C.c_void_p, C.POINTER(SurfaceRenderData)]),
    ("cn_solver_read_particles", C.c_int, [C.c_void_p, P_f32, P_f32, P_f32, u32]),
    ("cn_solver_write_particles", C.c_int, [C.c_void_p, P_f32, P_f32, u32]),
    ("cn_solver_read_strand_orientations", C.c_int, [C.c_void_p, P_f32, u32]),
    ("cn_solver_set_debug", C.c_int, [C.c_void_p, u32]),
    ("cn_solver_set_timing", C.c_int, [C.c_void_p, u32]),
    ("cn_solver_kernel_times", C.c_int, [C.c_void_p, C.c_void_p, u32, P_u32]),
    ("cn_solver_graph_stats", C.c_int, [C.c_void_p, P_u32, P_u32]),
    ("cn_solver_schedule_info", C.c_int, [C.c_void_p, C.POINTER(ScheduleInfo)]),
    ("cn_colour_constraints", C.c_int, [P_u32, u32, u32, u32, P_u32, P_u32, u32, P_u32]),
    ("cn_world_particle_layout_mapping", C.c_int, [C.c_void_p, C.POINTER(ParticleLayoutMapping)]),
    ("cn_sort_cell_keys_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, u32, C.c_void_p, C.c_void_p]),
    ("cn_solver_debug_read", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    ("cn_batch_desc_defaults", None, [C.POINTER(BatchDesc)]),
    ("cn_batch_create", C.c_int, [C.POINTER(BatchDesc), C.c_int, C.POINTER(C.c_void_p)]),
    ("cn_batch_destroy", None, [C.c_void_p]),
    ("cn_batch_add_scene", C.c_int, [C.c_void_p, C.POINTER(WorldSoA), P_u32]),
    ("cn_batch_remove_scene", C.c_int, [C.c_void_p, u32]),
    ("cn_batch_set_kinematic_target", C.c_int, [C.c_void_p, u32, u32, P_f32, P_f32]),
    ("cn_batch_step", C.c_int, [C.c_void_p, P_u32, u32, f32, C.c_void_p]),
    ("cn_batch_read_particles", C.c_int, [C.c_void_p, u32, P_f32, P_f32, u32]),
    ("cn_batch_export_scene", C.c_int, [C.c_void_p, u32, C.POINTER(WorldSoA)]),
    ("cn_batch_get_stats", C.c_int, [C.c_void_p, C.POINTER(BatchStats)]),
    ("cn_batch_set_schedule", C.c_int, [C.c_void_p, u32, u32]),
    ("cn_batch_set_fused", C.c_int, [C.c_void_p, u32]),
    ("cn_batch_set_xpbd_schedule", C.c_int, [C.c_void_p, u32]),
    ("cn_batch_autotune", C.c_int, [C.c_void_p, P_u32, u32, f32, C.POINTER(BatchTuning)]),
    ("cn_solver_export_dlpack", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    ("cn_solver_update_world", C.c_int, [C.c_void_p, C.POINTER(WorldSoA), u32]),
    ("cn_diff_desc_defaults", None, [C.POINTER(DiffDesc)]),
    ("cn_diff_create", C.c_int, [C.POINTER(DiffDesc), C.c_int, C.POINTER(C.c_void_p)]),
    ("cn_diff_destroy", None, [C.c_void_p]),
    ("cn_diff_set_scene", C.c_int, [C.c_void_p, C.POINTER(WorldSoA)]),
    ("cn_diff_forward", C.c_int, [C.c_void_p] + [C.c_void_p] * 6),
    ("cn_diff_backward", C.c_int, [C.c_void_p] + [C.c_void_p] * 6),
    ("cn_diff_memory", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("cn_server_desc_defaults", None, [C.POINTER(ServerDesc)]),
    ("cn_server_create", C.c_int, [C.c_void_p, C.POINTER(ServerDesc), u32, C.POINTER(C.c_void_p)]),
    ("cn_server_destroy", None, [C.c_void_p]),
    ("cn_server_register_scene", C.c_int, [C.c_void_p, C.POINTER(WorldSoA), P_u32]),
    ("cn_server_admit", C.c_int, [C.c_void_p, u32]),
    ("cn_server_submit", C.c_int, [C.c_void_p, u32, u32, u32, P_f32, C.POINTER(u64)]),
    ("cn_server_tick", C.c_int, [C.c_void_p, C.c_void_p, P_u32]),
    ("cn_server_drain", C.c_int, [C.c_void_p, C.c_void_p]),
    ("cn_server_poll", C.c_int, [C.c_void_p, C.POINTER(RequestDone), u32, P_u32]),
    ("cn_server_get_stats", C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    ("cn_server_read_particles", C.c_int, [C.c_void_p, u32, P_f32, P_f32, u32]),
]

_lib = None


def load(path: os.PathLike | str | None = None) -> C.CDLL:
    """Loads libcn_physics.so.  Raises if the library is missing: there is no fallback path."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python cressim-neo_b200/build.py`")
    lib = C.CDLL(str(p))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
