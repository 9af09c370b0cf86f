/*
 * cn_physics.h -- C ABI of the B200-native CRESSim-Neo particle physics substep.
 *
 * This header is the drop-in boundary for the particle substep that
 * cressim::neo::physics::PhysicsSolver runs
 * (reference: include/physics/physics_solver.h:150-205,
 *  src/physics/physics_solver.cpp:336-1401).  Every entry point takes plain
 * pointers and sizes; no C++ or torch types cross it.  Every call returns a
 * cn_status; cn_last_error() returns the message of the last failure on the
 * calling thread.
 *
 * Record layouts (cn_soft_edge, cn_soft_tet, ...) are byte-compatible with the
 * reference's GPU records (assets/shaders/include/physics/particle/
 * physics_particle_types.hlsli:111-290) so a caller that already packs the
 * reference's PhysicsWorld SoA can hand the same arrays over unchanged.
 */
#ifndef CN_PHYSICS_H
#define CN_PHYSICS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define CN_API __declspec(dllexport)
#else
#define CN_API __attribute__((visibility("default")))
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                              */
/* ------------------------------------------------------------------------ */
typedef enum cn_status {
    CN_OK = 0,
    CN_ERR_INVALID_ARGUMENT = 1,
    CN_ERR_CUDA = 2,
    CN_ERR_OUT_OF_MEMORY = 3,
    CN_ERR_NOT_INITIALIZED = 4,
    CN_ERR_CAPACITY = 5,     /* a fixed-capacity table overflowed */
    CN_ERR_NO_DEVICE = 6,
    CN_ERR_DEVICE_TIMEOUT = 7, /* a bounded device-side wait gave up */
    CN_ERR_UNSUPPORTED = 8
} cn_status;

/* Message of the last failing call on this thread ("" when none). */
CN_API const char *cn_last_error(void);
/* Library version string. */
CN_API const char *cn_version(void);

/* ------------------------------------------------------------------------ */
/* Solver settings: field-for-field mirror of PhysicsSolverDesc and its five  */
/* 32-byte settings structs (include/physics/physics_solver.h:22-143).        */
/* ------------------------------------------------------------------------ */
typedef struct cn_contact_settings {
    float slop;                                 /* 1e-3  */
    float manifold_merge_slop_multiplier;       /* 4     */
    float soft_relaxation;                      /* 0.95  */
    float soft_max_correction_per_iteration;    /* 0.05  */
    float restitution_velocity_threshold;       /* 0.5   */
    float restitution_penetration_slop_multiplier; /* 2  */
    float rigid_restitution_velocity_threshold; /* 0     */
    float position_friction_min_distance;       /* 1e-5  */
} cn_contact_settings;

typedef struct cn_rigid_settings {
    float depenetration_baumgarte;
    float depenetration_relaxation;
    float depenetration_max_correction_per_iteration;
    float velocity_penetration_stiffness;
    float max_translation_correction_per_iteration;
    float max_rotation_correction_per_iteration;
    float max_linear_velocity_correction_per_iteration;
    float max_angular_velocity_correction_per_iteration;
} cn_rigid_settings;

typedef struct cn_joint_settings {
    float ball_relaxation;
    float articulated_relaxation;
    float max_error;
    float max_translation_correction;
    float max_angular_correction;
    float regularization;
    float angular_regularization;
    float min_xpbd_dt;
} cn_joint_settings;

/* XPBD projection schedule of the soft families (edges, strand segments, bends and dihedrals,
 * strand joints, strand distances, tets; the family order of physics_solver.cpp:915-1019).
 *   CN_XPBD_GATHER: the reference's Jacobi solve -- every constraint of a family writes its
 *     correction records from the positions at the family's start, then each particle gathers
 *     its records in ascending constraint order.  The default; bit-exact with the reference.
 *   CN_XPBD_COLOUR_JACOBI: the same Jacobi update without the gather: each family is split by a
 *     greedy graph colouring (no two constraints of a colour share a particle or, for joints, a
 *     segment) and each colour adds its corrections straight into a per-particle sum, so the
 *     sum runs in colour order instead of constraint order (agrees with GATHER to rounding).
 *   CN_XPBD_COLOUR_GAUSS_SEIDEL: opt-in; each colour's corrections are applied before the next
 *     colour is solved (not the reference's update: stable at internal_relaxation 1, where the
 *     Jacobi gather diverges, and closer to the converged state after the same iterations). */
enum { CN_XPBD_GATHER = 0, CN_XPBD_COLOUR_JACOBI = 1, CN_XPBD_COLOUR_GAUSS_SEIDEL = 2 };
/* Fused iterations (opt-in): scenes of soft bodies against static or kinematic colliders (no
 * fluid, no particle-particle contacts, no dynamic bodies) small enough for one thread-block
 * cluster run all iterations of a substep in one cluster kernel, its phases separated by cluster
 * barriers (the same arithmetic, in the same order, as the per-phase kernels: bit-identical).
 * Off by default: on B200 the per-phase kernels over all SMs are faster even for a 4,096-particle
 * cube, whose dependent record -> position loads one 16-SM cluster cannot hide. */
enum { CN_FUSED_OFF = 0, CN_FUSED_ON = 1 };

typedef struct cn_soft_settings {
    float internal_relaxation; /* 0.2 */
    uint32_t xpbd_schedule;    /* CN_XPBD_GATHER */
    uint32_t fused_iterations; /* CN_FUSED_OFF */
    float reserved[5];
} cn_soft_settings;

typedef struct cn_fluid_settings {
    float constraint_relaxation;  /* 0.7  (kFluidSolveCoefficient) */
    float position_relaxation;    /* 1.0  (kFluidRelaxationFactor) */
    float boundary_density_scale; /* 0.12 */
    float boundary_delta_scale;   /* 0.08 */
    float max_under_density_ratio;/* 0.0  */
    float reserved[3];
} cn_fluid_settings;

typedef struct cn_solver_desc {
    float gravity[3];                 /* (0,-9.81,0) */
    uint32_t substeps;                /* >= 1 */
    uint32_t default_iterations;      /* 20 */
    uint32_t fluid_iterations;        /* 0 = default_iterations */
    uint32_t soft_internal_iterations;/* 0 = default_iterations */
    uint32_t soft_contact_iterations; /* 0 = default_iterations */
    uint32_t rigid_joint_iterations;  /* 0 = default_iterations */
    uint32_t rigid_rigid_contact_iterations; /* 0 = default_iterations */
    cn_contact_settings contact;
    cn_rigid_settings rigid;
    cn_joint_settings joints;
    cn_soft_settings soft;
    cn_fluid_settings fluid;
    uint32_t enable_blocking_readback; /* 1: step() copies x and v back into the synced host arrays */
    uint32_t max_fluid_neighborhood;   /* 128 (kDefaultFluidMaxNeighborhood) */
    /* Particle-rigid candidate pairs (and proxy contact slots) per particle: 8, the reference's
     * fixed rate (max(particles x 8, 64), physics_scene_gpu_state.cpp:726-727); 0 reads as 8.  No
     * reference counterpart as a setting: raise it for scenes whose particles touch more
     * colliders, where cn_solver_validate_meta reports the overflow. */
    uint32_t particle_rigid_pairs_per_particle;
} cn_solver_desc;

/* Fills the reference's defaults (physics_solver.h:22-143). */
CN_API void cn_solver_desc_defaults(cn_solver_desc *desc);

/* ------------------------------------------------------------------------ */
/* Device records (byte-compatible with physics_particle_types.hlsli and     */
/* physics_rigid_types.hlsli).                                               */
/* ------------------------------------------------------------------------ */
typedef struct cn_soft_edge {          /* GpuSoftEdge, 32 B */
    uint32_t particle_a, particle_b;
    float rest_length, compliance;
    uint32_t enabled, reserved0, reserved1, reserved2;
} cn_soft_edge;

typedef struct cn_soft_tet {           /* GpuSoftTet, 32 B */
    uint32_t particle_indices[4];
    float rest_volume, compliance;
    uint32_t reserved0, reserved1;
} cn_soft_tet;

typedef struct cn_soft_bend {          /* GpuSoftBend, 32 B */
    uint32_t particle0, particle1, particle2;
    float rest_angle, compliance;
    uint32_t reserved0, reserved1, reserved2;
} cn_soft_bend;

typedef struct cn_cloth_dihedral {     /* GpuClothDihedral, 32 B */
    uint32_t edge_particle0, edge_particle1, opposite_particle0, opposite_particle1;
    float rest_angle, compliance;
    uint32_t reserved0, reserved1;
} cn_cloth_dihedral;

typedef struct cn_strand_segment {     /* GpuStrandSegment, 32 B */
    uint32_t particle_a, particle_b;
    float rest_length, stretch_shear_compliance;
    float rest_orientation[4];         /* quaternion (x,y,z,w) */
} cn_strand_segment;

typedef struct cn_strand_joint {       /* GpuStrandJoint, 32 B */
    uint32_t segment_a, segment_b;
    float bend_compliance, twist_compliance;
    float rest_relative_orientation[4];
} cn_strand_joint;

typedef struct cn_strand_distance {    /* GpuStrandDistanceConstraint, 16 B */
    uint32_t particle_a, particle_b;
    float rest_length, distance_compliance;
} cn_strand_distance;

typedef struct cn_fluid_material {     /* GpuFluidMaterial / FluidMaterialGpu, 48 B */
    float rest_density, inv_rest_density, smoothing_radius, density_constraint_scale;
    float viscosity, cohesion, cohesion1, cohesion2;
    float surface_tension, vorticity_confinement, gravity_scale, cfl_radius;
} cn_fluid_material;

typedef struct cn_collider_geometry {  /* GpuColliderGeometryData, 48 B */
    float shape_params[4];             /* sphere: r; box: half extents; capsule: r, half height */
    float local_position[4];
    float local_orientation[4];
} cn_collider_geometry;

typedef struct cn_collider_broadphase { /* GpuColliderBroadPhaseData, 32 B */
    uint32_t owner_body, shape_type, environment_index, collision_layer;
    uint32_t collision_mask, enabled_flag, reserved1, reserved2;
} cn_collider_broadphase;

enum { CN_COLLIDER_SPHERE = 0, CN_COLLIDER_BOX = 1, CN_COLLIDER_CAPSULE = 2 };
enum { CN_BODY_STATIC = 0, CN_BODY_KINEMATIC = 1, CN_BODY_DYNAMIC = 2 };
enum { CN_PARTICLE_SOLID = 0, CN_PARTICLE_FLUID = 1 };
enum { CN_OWNER_NONE = 0, CN_OWNER_SOFT_BODY = 1, CN_OWNER_FLUID = 2, CN_OWNER_STRAND = 3,
       CN_OWNER_RIGID_BODY = 4, CN_OWNER_CLOTH = 5 };
#define CN_PHASE_GROUP_MASK 0x7fffffffu
#define CN_PHASE_SELF_COLLIDE 0x80000000u

/* ------------------------------------------------------------------------ */
/* World SoA: the host arrays PhysicsSolver::syncWorldState uploads           */
/* (reference: physics_types.h:696-920, physics_scene_gpu_state.cpp:2348).    */
/* All pointers are host pointers; arrays of length 0 may be NULL.            */
/* ------------------------------------------------------------------------ */
typedef struct cn_world_soa {
    /* particles */
    uint32_t particle_count;
    float *positions_inv_mass;      /* float4[N] xyz + invMass (read; written back on blocking readback) */
    float *velocities;              /* float4[N] */
    const float *radii;             /* float[N] */
    const uint32_t *kinds;          /* uint[N]  CN_PARTICLE_* */
    const uint32_t *metadata;       /* uint4[N] (environment, phase, collision layer, collision mask) */
    const uint32_t *material_indices;       /* uint[N] -> contact_materials */
    const uint32_t *fluid_material_indices; /* uint[N] -> fluid_materials (0xffffffff for solids) */
    const uint32_t *owner_types;    /* uint[N] CN_OWNER_* */
    const uint32_t *owner_indices;  /* uint[N] */
    const uint32_t *adjacency_offsets; /* uint[N] */
    const uint32_t *adjacency_counts;  /* uint[N] */
    const uint32_t *adjacency_indices; /* uint[adjacency_index_count] */
    uint32_t adjacency_index_count;
    float particle_grid_cell_size;  /* PhysicsWorld::particleGridCellSize() */

    uint32_t contact_material_count;
    const float *contact_materials; /* float4[] (friction, restitution, damping, staticFriction) */
    uint32_t fluid_material_count;
    const cn_fluid_material *fluid_materials;

    /* soft constraints */
    uint32_t edge_count;         const cn_soft_edge *edges;
    uint32_t bend_count;         const cn_soft_bend *bends;
    uint32_t dihedral_count;     const cn_cloth_dihedral *dihedrals;
    uint32_t tet_count;          const cn_soft_tet *tets;
    uint32_t strand_segment_count; const cn_strand_segment *strand_segments;
    float *strand_segment_orientations; /* float4[segments]: GpuStrandSegmentState */
    uint32_t strand_joint_count; const cn_strand_joint *strand_joints;
    uint32_t strand_distance_count; const cn_strand_distance *strand_distances;

    /* rigid bodies (static and kinematic bodies take part in the particle path) */
    uint32_t rigid_body_count;
    const float *body_positions_inv_mass;   /* float4[B] */
    const float *body_orientations;         /* float4[B] */
    const float *body_linear_velocities;    /* float4[B] */
    const float *body_angular_velocities;   /* float4[B] */
    const float *body_scales;               /* float4[B] */
    const float *body_inverse_inertia;      /* float4[B] */
    const uint32_t *body_types;             /* uint[B] CN_BODY_* */
    const float *body_kinematic_target_positions;    /* float4[B] */
    const float *body_kinematic_target_orientations; /* float4[B] */
    const uint32_t *body_kinematic_target_flags;     /* uint[B] bit0 = target enabled */
    const uint32_t *body_collider_ranges;   /* uint2[B] (offset, count) into body_collider_indices */
    const uint32_t *body_collider_indices;  /* uint[body_collider_index_count] */
    uint32_t body_collider_index_count;

    uint32_t collider_count;
    const cn_collider_geometry *collider_geometry;
    const cn_collider_broadphase *collider_broadphase;
    const float *collider_materials;        /* float4[C] (friction, restitution, 0, staticFriction) */

    /* surface render passes (skinning, normals, bounds); NULL: none */
    const struct cn_surface_render_data *surface_render;

    /* rigid proxy particles (PhysicsWorld packs them first: particles owned by a rigid body,
     * owner type CN_OWNER_RIGID_BODY, must form the prefix [0, proxies) of the particle order).
     * NULL when the world has none. */
    const float *rigid_proxy_local_positions;  /* float4[N]: scaled body-frame position (others 0) */
    const float *body_proxy_contact_materials; /* float4[B]: the proxies' packed contact material */
} cn_world_soa;

/* ------------------------------------------------------------------------ */
/* Surface render data: what PhysicsWorld::setSurfaceDeformableRenderData   */
/* holds (physics_world.cpp:3368; SurfaceDeformableRenderDataHost,           */
/* physics_types.h:1350-1392).  Every frame the solver skins the render      */
/* vertices, computes triangle and vertex normals and the per-surface world  */
/* AABBs from the particle positions (shaders in physics/soft/render/).     */
/* ------------------------------------------------------------------------ */
typedef struct cn_surface_vertex_binding {   /* SurfaceRenderVertexBinding (32 B) */
    uint32_t particle_indices[4];
    float weights[4];
} cn_surface_vertex_binding;
typedef struct cn_surface_triangle_range {   /* SurfaceRenderVertexTriangleRange (16 B) */
    uint32_t start, count, reserved0, reserved1;
} cn_surface_triangle_range;
typedef struct cn_surface_render_data {
    uint32_t vertex_count;
    const cn_surface_vertex_binding *vertex_bindings;          /* [vertex_count] */
    const float *fallback_normals;                             /* float4[vertex_count] */
    const cn_surface_triangle_range *vertex_triangle_ranges;   /* [vertex_count] */
    uint32_t vertex_triangle_index_count;
    const uint32_t *vertex_triangle_indices;                   /* incident triangles, in range order */
    uint32_t triangle_count;
    const uint32_t *triangle_particle_indices;                 /* uint4[triangle_count] (a, b, c, 0) */
    uint32_t surface_count;
    const uint32_t *surface_particle_ranges;                   /* uint2[surface_count] (offset, count) */
} cn_surface_render_data;

/* ------------------------------------------------------------------------ */
/* Host authoring (PhysicsWorld mirror): regular-grid soft bodies, fluid      */
/* lattices, cloth grids, strands, rigid bodies and colliders.  The world     */
/* derives the same state the reference derives at upload time.              */
/* ------------------------------------------------------------------------ */
typedef struct cn_world cn_world;

typedef struct cn_transform { float position[3]; float rotation[4]; float scale[3]; } cn_transform;

typedef struct cn_contact_material_desc {  /* ParticleContactMaterialDesc */
    float friction, restitution, damping, static_friction; /* static < 0 reuses friction */
} cn_contact_material_desc;

typedef struct cn_soft_body_grid_desc {   /* SoftBodyState with a RegularGrid source */
    float size[3];
    float target_particle_spacing;
    cn_transform rest_transform;
    float particle_mass;          /* 1.0 */
    float particle_radius;        /* 0.125 */
    float edge_compliance;
    float volume_compliance;
    uint32_t self_collision_enabled;
    uint32_t environment_index;
    uint32_t collision_layer, collision_mask;
    cn_contact_material_desc material;
    const uint32_t *static_particle_indices; uint32_t static_particle_count;
} cn_soft_body_grid_desc;

typedef struct cn_fluid_grid_desc {       /* FluidState with a RegularGrid source */
    float size[3];
    float target_particle_spacing;
    cn_transform rest_transform;
    float particle_mass;
    float particle_radius;
    float viscosity, cohesion, surface_tension, vorticity_confinement, gravity_scale, cfl_coefficient;
    uint32_t environment_index;
    uint32_t collision_layer, collision_mask;
    cn_contact_material_desc material;
} cn_fluid_grid_desc;

typedef struct cn_cloth_grid_desc {       /* ClothState with a rectangular grid source */
    uint32_t resolution[2];
    float size[2];
    cn_transform rest_transform;
    float particle_mass, particle_radius;
    float structural_compliance, bend_compliance;
    uint32_t self_collision_enabled, environment_index, collision_layer, collision_mask;
    cn_contact_material_desc material;
    const uint32_t *static_particle_indices; uint32_t static_particle_count;
} cn_cloth_grid_desc;

typedef struct cn_strand_desc {           /* StrandState */
    const float *rest_positions; uint32_t rest_position_count; /* float3[] */
    float particle_mass, particle_radius;
    float stretch_shear_compliance, bend_compliance, twist_compliance, distance_compliance;
    uint32_t self_collision_enabled, environment_index, collision_layer, collision_mask;
    cn_contact_material_desc material;
    const uint32_t *static_particle_indices; uint32_t static_particle_count;
} cn_strand_desc;

typedef struct cn_rigid_body_desc {
    uint32_t body_type;           /* CN_BODY_* */
    float position[3];
    float orientation[4];
    float scale[3];
    float mass;
    float inverse_inertia_local[3];
} cn_rigid_body_desc;

typedef struct cn_collider_desc {         /* ColliderState */
    uint32_t body;
    uint32_t shape_type;          /* CN_COLLIDER_* */
    float shape_params[4];
    float local_position[3];
    float local_orientation[4];
    uint32_t enabled;
    float friction, static_friction, restitution;
    uint32_t environment_index, collision_layer, collision_mask;
} cn_collider_desc;

CN_API void cn_soft_body_grid_desc_defaults(cn_soft_body_grid_desc *d);
CN_API void cn_fluid_grid_desc_defaults(cn_fluid_grid_desc *d);
CN_API void cn_cloth_grid_desc_defaults(cn_cloth_grid_desc *d);
CN_API void cn_strand_desc_defaults(cn_strand_desc *d);
/* Proxy collision particles of a rigid body (RigidBodyState proxy fields,
 * physics_types.h:401-417): spheres of one radius at body-frame points, carried with the body
 * every substep (physics_particle_sync_rigid_proxy_particles.cs.hlsl).  They collide with
 * particles (explicit contacts, whose share goes to the body) and with other bodies' colliders
 * (rigid contacts, physics_rigid_generate_proxy_contacts.cs.hlsl). */
typedef struct cn_rigid_proxy_desc {
    uint32_t body;
    const float *local_positions; uint32_t count;  /* float3[count], body frame before scaling */
    float radius;                                   /* <= 0: no proxies (the reference skips the body) */
    cn_contact_material_desc material;
    uint32_t environment_index;
    uint32_t collision_layer, collision_mask;       /* 1, 0xffffffff */
} cn_rigid_proxy_desc;

CN_API void cn_rigid_body_desc_defaults(cn_rigid_body_desc *d);
CN_API void cn_collider_desc_defaults(cn_collider_desc *d);
CN_API void cn_rigid_proxy_desc_defaults(cn_rigid_proxy_desc *d);

CN_API cn_status cn_world_create(cn_world **out_world);
CN_API void cn_world_destroy(cn_world *world);
/* reference: PhysicsWorld::upsertSoftBody + buildRegularGridSource (soft_body_authoring.cpp:81-176) */
CN_API cn_status cn_world_add_soft_body_grid(cn_world *w, const cn_soft_body_grid_desc *d, uint32_t *out_index);
/* SoftBodyState with a TetMesh source (soft_body_authoring.cpp:254-258): object-space positions
 * (xyz per vertex) and 4 indices per tetrahedron.  The grid fields size / target_particle_spacing
 * of `d` are ignored; transform, mass, radius, compliances, collision and static indices apply. */
CN_API cn_status cn_world_add_soft_body_tet_mesh(cn_world *w, const cn_soft_body_grid_desc *d, const float *positions,
                                                 uint32_t vertex_count, const uint32_t *tet_indices,
                                                 uint32_t tet_count, uint32_t *out_index);
/* SoftBodyState with a TetGenFiles source: the .node / .ele pair read as loadTetGenFiles does
 * (tetgen_loader.cpp:68-215); element rows must name node ids of the .node file. */
CN_API cn_status cn_world_add_soft_body_tetgen(cn_world *w, const cn_soft_body_grid_desc *d, const char *node_file,
                                               const char *ele_file, uint32_t *out_index);
/* SoftBodyState with a MeshfreeParticles source: distance edges to each particle's
 * neighbour_count nearest particles (buildMeshfreeKNearestGraph, soft_body_authoring.cpp:179-226). */
CN_API cn_status cn_world_add_soft_body_meshfree(cn_world *w, const cn_soft_body_grid_desc *d, const float *positions,
                                                 uint32_t particle_count, uint32_t neighbour_count, uint32_t *out_index);
/* reference: prepareFluidStateForInsert (physics_world.cpp:6857-6891), toFluidSolverMaterial (:191-262) */
CN_API cn_status cn_world_add_fluid_grid(cn_world *w, const cn_fluid_grid_desc *d, uint32_t *out_index);
CN_API cn_status cn_world_add_cloth_grid(cn_world *w, const cn_cloth_grid_desc *d, uint32_t *out_index);
CN_API cn_status cn_world_add_strand(cn_world *w, const cn_strand_desc *d, uint32_t *out_index);
CN_API cn_status cn_world_add_rigid_body(cn_world *w, const cn_rigid_body_desc *d, uint32_t *out_body);
CN_API cn_status cn_world_add_collider(cn_world *w, const cn_collider_desc *d, uint32_t *out_collider);
/* Sets (replaces) the proxy particles of body d->body; packed before every soft body, cloth,
 * strand and fluid particle, bodies in index order (physics_world.cpp:4931-5023). */
CN_API cn_status cn_world_set_rigid_proxy_particles(cn_world *w, const cn_rigid_proxy_desc *d);
/* A render mesh bound to a soft body or cloth, as the engine's World builds the surface render
 * data (world.cpp:3255-3554): every soft body and cloth gets a surface particle range (packed
 * [soft bodies][cloths]); the mesh's vertices are bound to the owner's particles -- one matching
 * rest particle within match_epsilon (makeExactSurfaceDeformableVertexBinding; cloth vertices must
 * match exactly one particle), or, for a meshfree soft body, the 4 nearest rest particles with
 * inverse-distance weights (makeNearestParticleSkinBinding) -- and each triangle to the dominant
 * particles of its vertices, with per-vertex incident-triangle lists in triangle order.  Mesh
 * positions are in the frame of the owner's authored rest positions (the reference's rest-local
 * frame); normals are the fallback normals (normalised; (0, 1, 0) when degenerate). */
enum { CN_SURFACE_OWNER_SOFT_BODY = 0, CN_SURFACE_OWNER_CLOTH = 1 };
typedef struct cn_surface_mesh_desc {
    uint32_t owner_kind;          /* CN_SURFACE_OWNER_* */
    uint32_t owner_index;         /* soft body / cloth index in authoring order */
    uint32_t vertex_count;
    const float *positions;       /* float3[vertex_count] */
    const float *normals;         /* float3[vertex_count] or NULL */
    uint32_t index_count;         /* 3 per triangle */
    const uint32_t *indices;
    float match_epsilon;          /* kSoftBodyVertexMatchEpsilon = 1e-3 */
    uint32_t reserved[3];
} cn_surface_mesh_desc;
CN_API void cn_surface_mesh_desc_defaults(cn_surface_mesh_desc *d);
/* out_first_vertex: index of the mesh's first render vertex in the packed render arrays. */
CN_API cn_status cn_world_add_surface_mesh(cn_world *w, const cn_surface_mesh_desc *d, uint32_t *out_first_vertex);
/* PhysicsWorld::setSurfaceDeformableRenderData: replaces the world's surface render data (and
 * the meshes added above) with a copy of `data`; NULL restores the built data. */
CN_API cn_status cn_world_set_surface_render(cn_world *w, const cn_surface_render_data *data);
/* Packs the SoA (PhysicsWorld::ensureDerivedStateUpToDate).  Pointers stay valid until the
 * next mutating call on the world; positions and velocities may be edited in place. */
CN_API cn_status cn_world_get_soa(cn_world *w, cn_world_soa *out);

/* ------------------------------------------------------------------------ */
/* Solver                                                                    */
/* ------------------------------------------------------------------------ */
typedef struct cn_solver cn_solver;

/* Device-side counters read by cn_solver_validate_meta
 * (reference: GpuParticleNeighborMeta, physics_particle_types.hlsli:49-64, and
 *  PhysicsSolver::validateGpuMetaBlocking, physics_solver.cpp:1403-1491). */
typedef struct cn_meta {
    uint32_t particle_rigid_candidate_count;
    uint32_t required_particle_rigid_candidate_count;
    uint32_t particle_rigid_candidate_overflow;
    uint32_t particle_particle_candidate_count;
    uint32_t required_particle_particle_candidate_count;
    uint32_t particle_particle_candidate_overflow;
    uint32_t fluid_boundary_candidate_overflow;  /* particles whose boundary candidates exceeded their capacity */
    uint32_t active_particle_rigid_contact_count;
    uint32_t active_particle_contact_count;
    uint32_t fluid_neighbor_truncations;         /* particles whose neighbour list hit max_fluid_neighborhood */
    uint32_t device_wait_timeouts;               /* bounded spins that gave up (sort look-back) */
    uint32_t rigid_rigid_candidate_count;        /* collider pairs of the rigid broadphase (GpuBroadPhaseMeta) */
    uint32_t required_rigid_rigid_candidate_count;
    uint32_t rigid_rigid_candidate_overflow;
    uint32_t proxy_rigid_contact_count;          /* proxy particle -> collider contacts (GpuProxyRigidContactMeta) */
    uint32_t required_proxy_rigid_contact_count;
    uint32_t proxy_rigid_contact_overflow;
    uint32_t reserved[1];
} cn_meta;

/* Non-owning device pointers (reference: PhysicsGpuSceneView,
 * include/physics/physics_gpu_scene_view.h:114-262).  Valid until
 * binding_generation changes. */
typedef struct cn_scene_view {
    void *positions_inv_mass;   /* float4[N] */
    void *previous_positions;   /* float4[N] */
    void *velocities;           /* float4[N] */
    void *radii;                /* float[N]  */
    void *kinds;                /* uint[N]   */
    void *edges; void *bends; void *dihedrals; void *tets;
    void *strand_segments; void *strand_joints; void *strand_distances; void *strand_segment_states;
    uint32_t particle_count, edge_count, bend_count, dihedral_count, tet_count;
    uint32_t strand_segment_count, strand_joint_count, strand_distance_count;
    uint64_t binding_generation;
    int32_t device;
    uint32_t reserved;
} cn_scene_view;

/* DLPack export of one scene-view buffer (the reference's shared_buffer_to_dlpack,
 * python/bindings.cpp:3303): a non-owning DLManagedTensor over the solver's device memory, valid
 * until binding_generation changes.  The struct layout is DLPack's (dlpack.h, version 0.8);
 * the consumer calls `deleter` when done.  Buffers: "positions_inv_mass", "previous_positions",
 * "velocities" (float32 N x 4), "radii" (float32 N), "kinds" (uint32 N), "strand_segment_states"
 * (float32 S x 4), "render_positions", "render_normals" (float32 V x 4), "surface_world_aabbs"
 * (float32 surfaces x 8: min xyzw, max xyzw). */
typedef struct cn_dl_tensor {
    void *data;
    int32_t device_type;            /* kDLCUDA = 2 */
    int32_t device_id;
    int32_t ndim;
    uint8_t dtype_code;             /* kDLInt 0, kDLUInt 1, kDLFloat 2 */
    uint8_t dtype_bits;
    uint16_t dtype_lanes;
    int64_t *shape;
    int64_t *strides;               /* NULL: compact row-major */
    uint64_t byte_offset;
} cn_dl_tensor;
typedef struct cn_dl_managed_tensor {
    cn_dl_tensor dl_tensor;
    void *manager_ctx;
    void (*deleter)(struct cn_dl_managed_tensor *self);
} cn_dl_managed_tensor;

/* PhysicsSolver(GpuDevice&, const PhysicsSolverDesc&) + initialize().  device: CUDA ordinal. */
CN_API cn_status cn_solver_create(const cn_solver_desc *desc, int device, cn_solver **out_solver);
CN_API void cn_solver_destroy(cn_solver *solver);
/* PhysicsSolver::syncWorldState: uploads the SoA, grows capacities, builds incidence tables. */
CN_API cn_status cn_solver_sync_world(cn_solver *solver, const cn_world_soa *world);
/* PhysicsSolver::step with FrameContext::deltaSeconds = frame_dt.  stream: cudaStream_t or NULL
 * (the solver's own stream).  With enable_blocking_readback the call waits and writes x and v back
 * into the synced host arrays. */
CN_API cn_status cn_solver_step(cn_solver *solver, float frame_dt, void *stream);
/* Runs `steps` frames back to back on the device (no per-frame host work when the scene is
 * capture-stable: the whole frame is one CUDA graph launch). */
CN_API cn_status cn_solver_step_many(cn_solver *solver, float frame_dt, uint32_t steps, void *stream);
/* PhysicsSolver::validateGpuMetaBlocking: waits for the device and reads the counters. */
CN_API cn_status cn_solver_validate_meta(cn_solver *solver, cn_meta *out_meta);
CN_API cn_status cn_solver_set_gravity(cn_solver *solver, float x, float y, float z);
/* Kinematic tool pose for the next step (reference: g_RigidBodyKinematicTarget*). */
CN_API cn_status cn_solver_set_kinematic_target(cn_solver *solver, uint32_t body,
                                                const float position[3], const float orientation[4]);
/* PhysicsSolver::gpuSceneView / softPositionsInvMassSharedBuffer: the native device buffers. */
CN_API cn_status cn_solver_scene_view(cn_solver *solver, cn_scene_view *out_view);
/* Surface render outputs (renderPositionsBuffer, renderNormalsBuffer, worldAabbsBuffer of
 * PhysicsGpuSoftSceneView, physics_gpu_scene_view.h:206-217), written at the end of every frame:
 * render positions float4 (xyz, 1), vertex normals float4 (xyz, 0), unnormalised triangle normals
 * float4, and AABBs as (min float4, max float4) pairs per 64-particle chunk and per surface. */
typedef struct cn_surface_render_view {
    void *render_positions;
    void *render_normals;
    void *triangle_normals;
    void *chunk_aabbs;
    void *world_aabbs;
    uint32_t vertex_count, triangle_count, chunk_count, surface_count;
    uint64_t binding_generation;
} cn_surface_render_view;
CN_API cn_status cn_solver_surface_render_view(cn_solver *solver, cn_surface_render_view *out_view);
/* Blocking host copies of the surface outputs (any pointer may be NULL): float4[vertex_count]
 * positions and normals, float4[2 * surface_count] world AABBs. */
CN_API cn_status cn_solver_read_surface_render(cn_solver *solver, float *positions, float *normals, float *world_aabbs);
CN_API cn_status cn_solver_export_dlpack(cn_solver *solver, const char *buffer, cn_dl_managed_tensor **out_tensor);
/* Incremental upload (the revision-counter path of uploadWorldState,
 * physics_scene_gpu_state.cpp:2348): the world's element counts must equal the synced ones;
 * the flagged categories are copied into the existing buffers, so device pointers and
 * binding_generation stay as they are. */
typedef enum cn_sync_flags {
    CN_SYNC_PARTICLE_STATE = 1,     /* positions / inverse masses, velocities */
    CN_SYNC_PARTICLE_ATTRIBUTES = 2,/* radii, metadata, material indices, contact / fluid materials;
                                     * refused when they change which contact or fluid terms run
                                     * (self-collision or solid groups, vorticity, cohesion / surface
                                     * tension) */
    CN_SYNC_CONSTRAINTS = 4,        /* edge, bend, dihedral, tet and strand records; their particle
                                     * (segment) indices must be the synced ones (else refused) */
    CN_SYNC_RIGID_BODIES = 8,       /* body poses, velocities, scales, inverse inertia, kinematic
                                     * targets; body types must be the synced ones (else refused) */
    CN_SYNC_COLLIDERS = 16,         /* collider geometry, broadphase records, materials; refused
                                     * when colliders are enabled, disabled or change bodies */
    CN_SYNC_SURFACE_RENDER = 32     /* surface render bindings, normals, triangles (same counts) */
} cn_sync_flags;
CN_API cn_status cn_solver_update_world(cn_solver *solver, const cn_world_soa *world, uint32_t flags);
/* Blocking copy of device particle state to host (readbackPredictedParticleStateBlocking).
 * Any pointer may be NULL. */
CN_API cn_status cn_solver_read_particles(cn_solver *solver, float *positions_inv_mass,
                                          float *velocities, float *previous_positions,
                                          uint32_t count);
/* Uploads particle positions and velocities only (host -> device, on the solver stream). */
CN_API cn_status cn_solver_write_particles(cn_solver *solver, const float *positions_inv_mass,
                                           const float *velocities, uint32_t count);
CN_API cn_status cn_solver_read_strand_orientations(cn_solver *solver, float *orientations,
                                                    uint32_t count);
/* Blocking copy of the rigid bodies' state after the last frame (readbackPredictedRigidStateBlocking,
 * physics_scene_gpu_state.h:423): float4[count] positions (w = inverse mass), orientations (xyzw),
 * linear and angular velocities.  Any pointer may be NULL. */
CN_API cn_status cn_solver_read_rigid_bodies(cn_solver *solver, float *positions_inv_mass, float *orientations,
                                             float *linear_velocities, float *angular_velocities, uint32_t count);
/* One frame with host state in and out (uploadParticles, physics_scene_gpu_state.cpp:3163, then
 * PhysicsSolver::step with its blocking readback, :4082-4155): float4[N] positions / velocities
 * are copied to the device (NULL: keep the device state), the frame runs, and the resulting
 * state is copied back (NULL: skip), all in order on `stream` (NULL: the solver's own) with one
 * wait at the end.  Host buffers should be pinned for full copy bandwidth. */
CN_API cn_status cn_solver_step_io(cn_solver *solver, float frame_dt, const float *positions_in,
                                   const float *velocities_in, float *positions_out, float *velocities_out,
                                   void *stream);

/* Debug switches (no reference counterpart; all off by default):
 *  CN_DEBUG_KEEP_FLUID_DELTA   keep the last iteration's packed fluid delta for cn_solver_debug_read;
 *  CN_DEBUG_POST_UPDATE_NEIGHBORS  rebuild fluid neighbour lists after the velocity update, as the
 *      reference does (physics_solver.cpp:1262-1268); the lists feed only vorticity confinement and
 *      render anisotropy, so the default schedule skips the rebuild;
 *  CN_DEBUG_FORCE_BROADPHASE   run the cell-key sort even when no consumer in the scene needs it
 *      (the reference always runs it once any contact family is enabled);
 *  CN_DEBUG_WALK_CELLS         build every fluid iteration's neighbour lists by walking the 27 cells,
 *      as the reference does, instead of filtering the substep's superset lists (same lists). */
enum { CN_DEBUG_KEEP_FLUID_DELTA = 1, CN_DEBUG_POST_UPDATE_NEIGHBORS = 2, CN_DEBUG_FORCE_BROADPHASE = 4,
       CN_DEBUG_WALK_CELLS = 8 };
CN_API cn_status cn_solver_set_debug(cn_solver *solver, uint32_t flags);

/* Per-kernel-group device times of the last replayed frame (no reference counterpart: the
 * reference records no GPU timestamps).  cn_solver_set_timing(1) records a CUDA event pair around
 * each kernel group of the captured frame; cn_solver_kernel_times sums them by group name. */
typedef struct cn_kernel_time {
    char name[32];
    float milliseconds;   /* summed over the group's launches in the last frame */
    uint32_t launches;    /* instances of the group in one frame */
} cn_kernel_time;
CN_API cn_status cn_solver_set_timing(cn_solver *solver, uint32_t enable);
CN_API cn_status cn_solver_kernel_times(cn_solver *solver, cn_kernel_time *out, uint32_t capacity,
                                        uint32_t *count);
/* Nodes of the captured frame graph: kernel launches and all nodes (launch count per frame). */
CN_API cn_status cn_solver_graph_stats(cn_solver *solver, uint32_t *kernel_nodes, uint32_t *nodes);

/* The XPBD schedule a synced solver runs (soft settings xpbd_schedule / fused_iterations). */
typedef struct cn_schedule_info {
    uint32_t xpbd_schedule;     /* CN_XPBD_* */
    uint32_t fused_iterations;  /* 1: each substep's iterations run in one cluster kernel */
    uint32_t cluster_ctas;      /* CTAs of that cluster (0 when not fused) */
    uint32_t threads_per_cta;
    uint32_t colours[6];        /* colours per family: edges, strand segments, bends + dihedrals,
                                 * strand joints, strand distances, tets (0 under CN_XPBD_GATHER) */
    uint32_t branches;          /* iteration work run concurrently on side streams (disjoint particles):
                                 * 1 the fluid chain, 2 the strand families, 4 the cloth bends */
} cn_schedule_info;
CN_API cn_status cn_solver_schedule_info(cn_solver *solver, cn_schedule_info *out);

/* Greedy graph colouring of one constraint family (host only, no device needed).  Constraint c,
 * taken in ascending order, receives the lowest colour that no earlier constraint sharing one of
 * its elements has.  elements[c * per_constraint + k] are constraint c's particles (segments for
 * strand joints); entries >= element_count are ignored.  Writes order[constraint_count] (the
 * constraints grouped by colour, ascending within a colour) and colour_starts[colours + 1];
 * *colours receives the colour count.  CN_ERR_CAPACITY when more than colour_capacity colours
 * are needed (colour_starts then holds colour_capacity + 1 entries at most). */
CN_API cn_status cn_colour_constraints(const uint32_t *elements, uint32_t constraint_count, uint32_t per_constraint,
                                       uint32_t element_count, uint32_t *order, uint32_t *colour_starts,
                                       uint32_t colour_capacity, uint32_t *colours);

/* Intermediate buffers of the last substep, for parity checks.  Each is converted to the
 * reference's layout and indexing (particle order, not cell order). */
typedef enum cn_debug_buffer {
    CN_DEBUG_CELL_ENTRIES = 0,     /* int4[N]: cellX, cellY, cellZ, cellKey (GpuParticleBroadPhaseEntry) */
    CN_DEBUG_SORTED_KEYS = 1,      /* uint2[N]: (cellKey, elementIdx) after the stable sort */
    CN_DEBUG_CELL_RANGES = 2,      /* uint4[nextPow2(2N)]: compacted (key, start, end, 0), rest key=0xffffffff */
    CN_DEBUG_FLUID_NEIGHBOR_COUNTS = 3, /* uint[N] */
    CN_DEBUG_FLUID_NEIGHBORS = 4,  /* uint[N * max_fluid_neighborhood]: neighbour particle indices */
    CN_DEBUG_FLUID_CONSTRAINTS = 5,/* float4[N]: surface normal xyz, density constraint w */
    CN_DEBUG_FLUID_DELTA = 6,      /* float4[N]: last packed delta + interaction weight */
    CN_DEBUG_RIGID_CONTACTS = 7,   /* 64 B records of the last iteration's particle-rigid contacts */
    CN_DEBUG_FLUID_SUPERSET_COUNTS = 8 /* uint[N]: candidates within h * 1.25 recorded at the substep's first
                                        * iteration (no reference counterpart; zeros when the lists are off) */
} cn_debug_buffer;
/* Copies at most capacity_bytes; *out_bytes receives the full size of the buffer. */
CN_API cn_status cn_solver_debug_read(cn_solver *solver, cn_debug_buffer which, void *dst,
                                      size_t capacity_bytes, size_t *out_bytes);

/* ------------------------------------------------------------------------ */
/* Batched scenes (no counterpart in the reference, which steps one          */
/* PhysicsWorld per PhysicsSolver).  Independent soft-tissue scenes (XPBD     */
/* edges + tets, static / kinematic colliders) live in one device pool, each  */
/* in its own index ranges, and any subset of them is stepped by one tick:    */
/* one CUDA graph whose kernels stride over per-scene work tiles.  A scene    */
/* stepped in a batch gets the same bits as in a cn_solver of its own under  */
/* the same XPBD schedule (solver.soft.xpbd_schedule: gather, or a coloured  */
/* schedule, for which the pool also holds each scene's colourings).         */
/* ------------------------------------------------------------------------ */
typedef struct cn_batch cn_batch;

typedef struct cn_batch_desc {
    cn_solver_desc solver;          /* substeps, iterations and settings shared by all scenes */
    uint64_t memory_budget_bytes;   /* admission bound: device bytes the admitted scenes may use */
    uint32_t max_scenes;            /* resident scenes at most (sizes the per-tick work lists) */
    uint32_t particle_capacity;     /* pool sizes; 0 = split from the budget by a soft-tissue mix */
    uint32_t edge_capacity, tet_capacity, body_capacity, collider_capacity;
    uint32_t tile_elements;         /* elements per work tile (autotuned by cn_batch_autotune) */
    uint32_t blocks_per_sm;         /* grid of the tile kernels = SMs x this */
    uint32_t rigid_pairs_per_particle;
    uint32_t fused_cluster_ctas;    /* 0: the iterations as per-phase kernels over the tick's work
                                     * lists; n: as one persistent kernel, each cluster of n CTAs
                                     * taking one scene at a time (bit-identical; autotuned) */
    uint32_t reserved[2];
} cn_batch_desc;

typedef struct cn_batch_stats {
    uint32_t resident_scenes;
    uint32_t particles_used, particle_capacity, edges_used, edge_capacity, tets_used, tet_capacity;
    uint32_t tile_elements, grid_blocks, fused_cluster_ctas;
    uint32_t xpbd_schedule, reserved0; /* the running XPBD schedule (CN_XPBD_*) */
    uint64_t budget_bytes, budget_used_bytes, pool_bytes, ticks;
} cn_batch_stats;

/* cluster_ctas: 0 for the per-phase iteration kernels, else the CTAs per scene of the persistent
 * fused iterations (cn_batch_desc.fused_cluster_ctas); xpbd_schedule: CN_XPBD_*. */
typedef struct cn_batch_candidate {
    uint32_t tile_elements, blocks_per_sm;
    float tick_ms;
    uint32_t cluster_ctas, xpbd_schedule;
} cn_batch_candidate;
typedef struct cn_batch_tuning {
    uint32_t tile_elements, blocks_per_sm;
    float tick_ms;
    uint32_t candidate_count;
    cn_batch_candidate candidates[24];
    uint32_t cluster_ctas, xpbd_schedule;
    uint32_t reserved[2];
} cn_batch_tuning;

CN_API void cn_batch_desc_defaults(cn_batch_desc *desc);
CN_API cn_status cn_batch_create(const cn_batch_desc *desc, int cuda_device, cn_batch **out_batch);
CN_API void cn_batch_destroy(cn_batch *batch);
/* Admits one scene (a world SoA with 0-based indices).  CN_ERR_CAPACITY when the budget or the
 * pool has no room; CN_ERR_UNSUPPORTED for fluid, cloth, strand, self-colliding or dynamic-body
 * content, and in a batch created with a coloured schedule for an edge or tet family that needs
 * more than 256 colours.  The upload is asynchronous: the scene's arrays go to the device in one transfer and
 * are scattered into its pool ranges on the batch's upload stream, which the next cn_batch_step
 * waits for; the SoA may be reused as soon as the call returns. */
CN_API cn_status cn_batch_add_scene(cn_batch *batch, const cn_world_soa *world, uint32_t *out_scene);
CN_API cn_status cn_batch_remove_scene(cn_batch *batch, uint32_t scene);
/* Staged until the next cn_batch_step, as cn_solver_set_kinematic_target for one scene's body. */
CN_API cn_status cn_batch_set_kinematic_target(cn_batch *batch, uint32_t scene, uint32_t body,
                                               const float position[3], const float orientation[4]);
/* One frame of every listed scene (the others do not move), asynchronous on `stream`. */
CN_API cn_status cn_batch_step(cn_batch *batch, const uint32_t *scenes, uint32_t count, float frame_dt,
                               void *stream);
CN_API cn_status cn_batch_read_particles(cn_batch *batch, uint32_t scene, float *positions_inv_mass,
                                         float *velocities, uint32_t count);
/* Writes a scene's particle and rigid-body state back into its SoA (before evicting it). */
CN_API cn_status cn_batch_export_scene(cn_batch *batch, uint32_t scene, cn_world_soa *world);
CN_API cn_status cn_batch_get_stats(cn_batch *batch, cn_batch_stats *out);
CN_API cn_status cn_batch_set_schedule(cn_batch *batch, uint32_t tile_elements, uint32_t blocks_per_sm);
/* 0: per-phase iteration kernels; 1, 2, 4 or 8: the persistent fused iterations with clusters of
 * that many CTAs.  CN_ERR_UNSUPPORTED when the device cannot form such clusters. */
CN_API cn_status cn_batch_set_fused(cn_batch *batch, uint32_t cluster_ctas);
/* The XPBD schedule of the next ticks: CN_XPBD_GATHER always; a coloured one only in a batch
 * created with a coloured schedule (CN_ERR_UNSUPPORTED otherwise) and with the per-phase kernels
 * (cluster_ctas 0). */
CN_API cn_status cn_batch_set_xpbd_schedule(cn_batch *batch, uint32_t schedule);
/* Times a tick of `scenes` for each (tile size, blocks per SM) candidate of the per-phase
 * kernels, then for the persistent fused iterations with clusters of 1, 2, 4 and 8 CTAs (at the
 * best tile schedule), keeps the fastest and restores the scenes' state.  In a batch created with
 * colour Jacobi it also times colour Jacobi at the best tile size (its results equal the gather
 * schedule's up to the order of each particle's sum, within 1e-5); under Gauss-Seidel, a
 * different iteration, only the tile candidates are timed, all under Gauss-Seidel. */
CN_API cn_status cn_batch_autotune(cn_batch *batch, const uint32_t *scenes, uint32_t count, float frame_dt,
                                   cn_batch_tuning *out);

/* Serving loop over a batch (no counterpart in the reference).  Scenes are registered once (a
 * host copy is kept) and admitted to the batch's pool when a request needs them and the memory
 * budget allows, evicting idle scenes (least recently stepped first) when it does not.  Each
 * tick steps one frame of every resident scene with pending work; requests that arrive while
 * ticks run join the next tick.  Times are seconds on the server's steady clock. */
typedef struct cn_server cn_server;
typedef struct cn_server_desc {
    float frame_dt;
    uint32_t max_scenes_per_tick;   /* 0 = every scene with pending work */
    uint32_t reserved[6];
} cn_server_desc;
typedef struct cn_request_done {
    uint64_t request_id;
    uint32_t scene, steps;
    double submit_s, first_tick_s, done_s;
} cn_request_done;
typedef struct cn_server_stats {
    uint64_t ticks, scene_steps, particle_substeps, admissions, evictions, completed, pending;
    uint32_t resident_scenes, registered_scenes;
    double gpu_ms;
    float tick_ms_p50, tick_ms_p99;
} cn_server_stats;

CN_API void cn_server_desc_defaults(cn_server_desc *desc);
/* `substeps` is the batch's substep count (used for the particle-substep count). */
CN_API cn_status cn_server_create(cn_batch *batch, const cn_server_desc *desc, uint32_t substeps, cn_server **out);
/* Removes the server's resident scenes from its batch: call it before cn_batch_destroy of that batch. */
CN_API void cn_server_destroy(cn_server *server);
CN_API cn_status cn_server_register_scene(cn_server *server, const cn_world_soa *world, uint32_t *out_scene);
/* Makes a registered scene resident ahead of its requests (evicting idle scenes if needed);
 * CN_ERR_CAPACITY when the budget has no room. */
CN_API cn_status cn_server_admit(cn_server *server, uint32_t scene);
/* k frames of one scene; tool_targets (k x 7 floats: position xyz, orientation xyzw) drive the
 * kinematic body `tool_body` frame by frame, or NULL. */
CN_API cn_status cn_server_submit(cn_server *server, uint32_t scene, uint32_t steps, uint32_t tool_body,
                                  const float *tool_targets, uint64_t *out_request);
/* Launches one tick (asynchronous on `stream`), then waits for the tick before it. */
CN_API cn_status cn_server_tick(cn_server *server, void *stream, uint32_t *out_stepped_scenes);
/* Ticks until no request is pending and every tick has finished. */
CN_API cn_status cn_server_drain(cn_server *server, void *stream);
CN_API cn_status cn_server_poll(cn_server *server, cn_request_done *out, uint32_t capacity, uint32_t *out_count);
CN_API cn_status cn_server_get_stats(cn_server *server, cn_server_stats *out);
CN_API cn_status cn_server_read_particles(cn_server *server, uint32_t scene, float *positions_inv_mass,
                                          float *velocities, uint32_t count);

/* ------------------------------------------------------------------------ */
/* Differentiable XPBD rollout (no counterpart in the reference).  The soft   */
/* substep (predict, Jacobi edge + tet iterations, velocity update) of a      */
/* scene without colliders, forward with checkpoints every                    */
/* checkpoint_interval substeps and a hand-written adjoint giving d loss /    */
/* d (per-tet compliance, initial positions, initial velocities).  Buffers are*/
/* device pointers of float (precision 4) or double (precision 8); positions  */
/* and velocities are 4 values per particle (xyz + invMass / unused).         */
/* ------------------------------------------------------------------------ */
typedef struct cn_diff cn_diff;
typedef struct cn_diff_desc {
    float gravity[3];
    uint32_t substeps;              /* substeps of one rollout */
    uint32_t iterations;            /* Jacobi iterations per substep */
    float substep_dt;
    float relaxation;               /* softInternalRelaxation (0.2) */
    uint32_t checkpoint_interval;   /* substeps between saved (x, v) states */
    uint32_t precision;             /* 4 = float, 8 = double */
    uint32_t reserved[4];
} cn_diff_desc;
CN_API void cn_diff_desc_defaults(cn_diff_desc *desc);
CN_API cn_status cn_diff_create(const cn_diff_desc *desc, int cuda_device, cn_diff **out);
CN_API void cn_diff_destroy(cn_diff *diff);
CN_API cn_status cn_diff_set_scene(cn_diff *diff, const cn_world_soa *world);
CN_API cn_status cn_diff_forward(cn_diff *diff, const void *tet_compliance, const void *x0, const void *v0,
                                 void *x_out, void *v_out, void *stream);
/* Adjoint of the last forward: grad_x_out / grad_v_out (either may be NULL = zero) in, the
 * gradients with respect to the forward's inputs out (grad_x0 / grad_v0 may be NULL). */
CN_API cn_status cn_diff_backward(cn_diff *diff, const void *grad_x_out, const void *grad_v_out,
                                  void *grad_tet_compliance, void *grad_x0, void *grad_v0, void *stream);
/* Device bytes of the state the adjoint keeps (checkpoints, one segment, one substep). */
CN_API cn_status cn_diff_memory(cn_diff *diff, uint64_t *bytes);

/* ParticleLayoutMapping (include/engine/particle_layout_mapping.h:11-68, filled by
 * Runtime::tryGetPreparedParticleLayoutMapping, src/engine/runtime.cpp:867-955): the packed
 * particle slots' owners and filters, and each owner's slot range, for the RL-environment glue
 * that slices the exported particle buffers.  Per-particle arrays hold particle_count entries,
 * per-owner arrays the owner count; owner ids are the handles the cn_world_add_* calls returned
 * (the reference's EntityId of the owning entity).  layout_revision changes whenever a new
 * packing changes how slots are interpreted.  Pointers stay valid until the next authoring call. */
typedef struct cn_particle_owner_ranges {
    uint32_t count;
    const uint64_t *ids;
    const uint32_t *environment_indices, *particle_offsets, *particle_counts;
} cn_particle_owner_ranges;

typedef struct cn_particle_layout_mapping {
    uint32_t particle_count, soft_body_count, cloth_count, fluid_count, strand_count;
    uint64_t layout_revision;
    const uint32_t *environment_indices, *particle_kinds, *owner_types, *owner_indices;
    const uint32_t *strand_ids, *strand_orders, *strand_roles, *owning_soft_body_indices;
    const uint32_t *particle_material_indices, *fluid_material_indices;
    const uint32_t *phases, *collision_layers, *collision_masks;
    const uint32_t *adjacency_offsets, *adjacency_counts;
    cn_particle_owner_ranges soft_bodies, cloths, fluids, strands;
} cn_particle_layout_mapping;

CN_API cn_status cn_world_particle_layout_mapping(cn_world *world, cn_particle_layout_mapping *out);

/* Allocation-free broadphase sort (no counterpart in the reference).
 * For callers that must not allocate device memory while they run -- engines whose device memory
 * belongs to their own pool, frame loops that cannot afford the allocator's implicit
 * synchronisation, real-time code that reserves everything up front.  Sorts `count` cell keys
 * stably (the permutation equals a stable sort by key, as the broadphase's) into caller-owned
 * device buffers: sorted_keys[i] is the i-th key, sorted_indices[i] its input position.
 * Limit: count <= 1048576; larger counts return CN_ERR_CAPACITY.  Scratch lives in a ~10 MiB
 * file-scope device array that every GPU loading the library keeps until exit; the first call on
 * a device looks its address up (cudaGetSymbolAddress), so make that first call before any stream
 * capture.  All calls share the array: calls that overlap on the GPU (different streams or
 * threads without ordering) race.  The cached address does not survive cudaDeviceReset: do not
 * call this on a device that has been reset.  `keys`, `sorted_keys` and `sorted_indices` each
 * hold `count` 32-bit words and must not alias one another (CN_ERR_INVALID_ARGUMENT); `keys` is
 * not modified.  `out_timeouts` (a device pointer, may be NULL) receives the number of look-back
 * waits that gave up; a nonzero value means the output permutation is invalid.  Outputs are
 * ready once `stream` (may be NULL) has completed the work this call enqueued. */
CN_API cn_status cn_sort_cell_keys_noalloc(const uint32_t *keys, uint32_t *sorted_keys,
                                           uint32_t *sorted_indices, uint32_t count,
                                           uint32_t *out_timeouts, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CN_PHYSICS_H */
