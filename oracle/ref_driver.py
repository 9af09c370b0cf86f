"""TEST INFRASTRUCTURE ONLY: runs the reference's own compute shaders on the CPU.

oracle/ref_build.py compiles the reference's HLSL kernels (CRESSim-Neo,
assets/shaders/physics/**) for the host into oracle/_ref/libcn_ref_shaders.so.  This module
binds host buffers to them and dispatches them in the order PhysicsSolver::step does
(src/physics/physics_solver.cpp:435-1310), with the buffer bindings of PhysicsPassDispatcher
(src/physics/physics_pass_dispatcher.cpp) and the dispatch constants of physics_solver.cpp:437-471.
Only the generator of the reference fixtures (tests/golden/make_ref_golden.py) uses it.

A few steps the reference runs as multi-pass GPU algorithms are computed here directly, with the
same results by construction:
  * the 32-pass stable split radix sort of the (cellKey, particleIndex) pairs
    (physics_pass_dispatcher.cpp:3963-4057) is a stable sort by key;
  * the block exclusive scans (physics_scan_block / physics_scan_add_offsets) are prefix sums;
  * the rigid broad-phase BVH (morton codes, radix sort, hierarchy and bounding-box passes) is
    replaced by a valid BVH over the same leaf boxes -- the collider AABBs that the reference's
    own physics_rigid_update_world_aabbs kernel writes -- shaped as a chain whose depth-first walk
    (right child first, as the candidate kernels' stacks pop) visits the colliders in ascending
    index order.  The candidate kernels then traverse it unchanged; their candidate sets are the
    reference's, in ascending collider order (moving colliders first, then static ones).

Scope: particles (soft bodies, cloth, strands, fluid) with static and kinematic rigid colliders.
Dynamic bodies, rigid proxies, joints and suturing are not driven here.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "libcn_ref_shaders.so"

KIND_FLUID = 1
BODY_STATIC, BODY_KINEMATIC, BODY_DYNAMIC = 0, 1, 2


class Kernel:
    def __init__(self, lib, name):
        self.name = name
        info = getattr(lib, name + "_info")
        info.restype = C.c_char_p
        parts = info().decode().split(";")
        self.numthreads = tuple(int(x) for x in parts[0].split("=")[1].split(","))
        self.buffers = {}
        self.constants = {}
        for p in parts[1:]:
            f = p.split(":")
            if f[0] == "buffer":
                self.buffers[f[1]] = f[2]
            elif f[0] == "const":
                self.constants[f[1]] = f[2]
        self._bind = getattr(lib, name + "_bind")
        self._bind.argtypes = [C.c_char_p, C.c_void_p, C.c_ulonglong]
        self._set = getattr(lib, name + "_set")
        self._set.argtypes = [C.c_char_p, C.c_void_p, C.c_ulonglong]
        self._dispatch = getattr(lib, name + "_dispatch")
        self._dispatch.argtypes = [C.c_uint, C.c_uint, C.c_uint]
        sz = getattr(lib, name + "_sizeof")
        sz.restype = C.c_ulonglong
        sz.argtypes = [C.c_char_p]
        self.sizes = {b: sz(b.encode()) for b in self.buffers}

    def run(self, mem: dict, consts: dict, threads: int, alias: dict | None = None):
        alias = alias or {}
        keep = []
        for var in self.buffers:
            key = alias.get(var, var)
            if key not in mem:
                raise KeyError(f"{self.name}: no buffer for {var} ({key})")
            arr = mem[key]
            assert arr.flags.c_contiguous
            if arr.nbytes % self.sizes[var]:
                raise ValueError(f"{self.name}: {var} has {arr.nbytes} bytes, element {self.sizes[var]}")
            rc = self._bind(var.encode(), arr.ctypes.data if arr.nbytes else None, arr.nbytes)
            if rc != 0:
                raise RuntimeError(f"{self.name}: bind {var} -> {rc}")
            keep.append(arr)
        for name, typ in self.constants.items():
            if name not in consts:
                continue
            v = consts[name]
            if typ == "float":
                b = np.array([v], np.float32)
            elif typ in ("uint", "int"):
                b = np.array([v], np.uint32 if typ == "uint" else np.int32)
            elif typ == "float4":
                b = np.asarray(v, np.float32).reshape(4)
            else:
                raise TypeError(f"{self.name}: constant {name} of type {typ}")
            rc = self._set(name.encode(), b.ctypes.data, b.nbytes)
            if rc != 0:
                raise RuntimeError(f"{self.name}: set {name} -> {rc}")
        groups = (int(threads) + self.numthreads[0] - 1) // self.numthreads[0]
        if groups:
            self._dispatch(groups, 1, 1)


class RefLib:
    def __init__(self):
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} is not built (python oracle/ref_build.py)")
        self.lib = C.CDLL(str(LIB))
        self.lib.cnref_out_of_range.restype = C.c_ulonglong
        self.lib.cnref_barrier_calls.restype = C.c_int
        self.kernels = {}

    def __getitem__(self, name) -> Kernel:
        if name not in self.kernels:
            self.kernels[name] = Kernel(self.lib, name)
        return self.kernels[name]

    def counters(self):
        return int(self.lib.cnref_out_of_range()), int(self.lib.cnref_barrier_calls())


def _view(ptr, count, dtype, width=1):
    if not ptr or count == 0:
        return np.zeros((count, width) if width > 1 else count, dtype)
    addr = C.cast(ptr, C.c_void_p).value
    nbytes = count * width * np.dtype(dtype).itemsize
    raw = (C.c_uint8 * nbytes).from_address(addr)
    a = np.frombuffer(raw, dtype=dtype).copy()
    return a.reshape(count, width) if width > 1 else a


def _records(ptr, count, size):
    return _view(ptr, count * size // 4, np.uint32).reshape(count, size // 4) if count else \
        np.zeros((0, size // 4), np.uint32)


def _incidence(n_owner: int, refs: list[list[tuple[int, int]]]):
    """GpuSoftConstraintRange per owner + incident records {index, slot, 0, 0} in list order
    (physics_scene_gpu_state.cpp:3255-3445, buildConstraintAdjacencyRanges)."""
    ranges = np.zeros((max(n_owner, 1), 4), np.uint32)
    flat = []
    for i, r in enumerate(refs):
        ranges[i, 0] = len(flat)
        ranges[i, 1] = len(r)
        flat.extend(r)
    inc = np.zeros((max(len(flat), 1), 4), np.uint32)
    for k, (idx, slot) in enumerate(flat):
        inc[k, 0] = idx
        inc[k, 1] = slot
    return ranges, inc


def _next_pow2(v: int) -> int:
    p = 1
    while p < v:
        p <<= 1
    return p


def _f(a):
    return np.ascontiguousarray(a, np.float32)


class RefSolver:
    """The reference's substep pipeline over one world SoA (cn_world_soa) and solver desc."""

    def __init__(self, desc, soa, pair_capacity_per_particle: int = 64):
        self.L = RefLib()
        self.desc = desc
        m = {}
        N = soa.particle_count
        self.N = N
        m["g_ParticlePositionsInvMass"] = _view(soa.positions_inv_mass, N, np.float32, 4)
        m["g_ParticlePreviousPositions"] = m["g_ParticlePositionsInvMass"].copy()
        m["g_ParticleVelocities"] = _view(soa.velocities, N, np.float32, 4)
        m["g_ParticleRadii"] = _view(soa.radii, N, np.float32)
        m["g_ParticleKinds"] = _view(soa.kinds, N, np.uint32)
        m["g_ParticleBroadPhaseMetadata"] = _view(soa.metadata, N, np.uint32, 4)
        m["g_ParticleMaterialIndices"] = _view(soa.material_indices, N, np.uint32)
        m["g_ParticleContactMaterials"] = _view(soa.contact_materials, max(soa.contact_material_count, 1), np.float32, 4)
        m["g_FluidMaterialIndices"] = _view(soa.fluid_material_indices, N, np.uint32)
        m["g_FluidMaterials"] = _records(soa.fluid_materials, max(soa.fluid_material_count, 1), 48)
        m["g_ParticleOwnerTypes"] = _view(soa.owner_types, N, np.uint32)
        m["g_ParticleOwnerIndices"] = _view(soa.owner_indices, N, np.uint32)
        m["g_ParticleAdjacencyOffsets"] = _view(soa.adjacency_offsets, N, np.uint32)
        m["g_ParticleAdjacencyCounts"] = _view(soa.adjacency_counts, N, np.uint32)
        m["g_ParticleAdjacencyIndices"] = _view(soa.adjacency_indices, max(soa.adjacency_index_count, 1), np.uint32)
        # Suturing is not driven: no strand roles, no links, every insertion state "outside".
        m["g_ParticleStrandRoles"] = np.zeros(N, np.uint32)
        m["g_SuturingNeighborLinks"] = np.full((N, 4), 0xFFFFFFFF, np.uint32)
        m["g_ParticleOwningSoftBodyIndices"] = np.full(N, 0xFFFFFFFF, np.uint32)
        m["g_SuturingInsertionStates"] = np.zeros((N, 12), np.uint32)
        m["g_RigidProxyLocalPositions"] = np.zeros((N, 4), np.float32)

        # soft topology (physics_particle_types.hlsli:111-290 records, unchanged)
        E, T, Bn, D = soa.edge_count, soa.tet_count, soa.bend_count, soa.dihedral_count
        S, J, Ds = soa.strand_segment_count, soa.strand_joint_count, soa.strand_distance_count
        self.counts = dict(E=E, T=T, Bn=Bn, D=D, S=S, J=J, Ds=Ds)
        m["g_SoftEdges"] = _records(soa.edges, max(E, 1), 32)
        m["g_SoftTets"] = _records(soa.tets, max(T, 1), 32)
        m["g_SoftBends"] = _records(soa.bends, max(Bn, 1), 32)
        m["g_ClothDihedrals"] = _records(soa.dihedrals, max(D, 1), 32)
        m["g_StrandSegments"] = _records(soa.strand_segments, max(S, 1), 32)
        m["g_StrandSegmentStates"] = _view(soa.strand_segment_orientations, max(S, 1), np.float32, 4) if S else \
            np.zeros((1, 4), np.float32)
        m["g_StrandJoints"] = _records(soa.strand_joints, max(J, 1), 32)
        m["g_StrandDistanceConstraints"] = _records(soa.strand_distances, max(Ds, 1), 16)
        m["g_SoftEdgeLambdas"] = np.zeros(max(E, 1), np.float32)
        m["g_SoftTetLambdas"] = np.zeros(max(T, 1), np.float32)
        m["g_BendLambdas"] = np.zeros(max(Bn + D, 1), np.float32)
        m["g_StrandSegmentLambdas"] = np.zeros((max(S, 1), 4), np.float32)
        m["g_StrandJointLambdas"] = np.zeros((max(J, 1), 4), np.float32)
        m["g_StrandDistanceLambdas"] = np.zeros(max(Ds, 1), np.float32)
        m["g_SoftEdgeCorrections"] = np.zeros((max(E, 1), 8), np.float32)
        m["g_SoftTetCorrections"] = np.zeros((max(T, 1), 16), np.float32)
        m["g_BendCorrections"] = np.zeros((max(Bn + D, 1), 16), np.float32)
        m["g_StrandSegmentCorrections"] = np.zeros((max(S, 1), 12), np.float32)
        m["g_StrandJointCorrections"] = np.zeros((max(J, 1), 20), np.float32)
        m["g_StrandDistanceCorrections"] = np.zeros((max(Ds, 1), 8), np.float32)
        # incidence tables in ascending constraint order (physics_scene_gpu_state.cpp:3270-3445)
        edges, tets = m["g_SoftEdges"], m["g_SoftTets"]
        refs = [[] for _ in range(N)]
        for e in range(E):
            refs[edges[e, 0]].append((e, 0))
            refs[edges[e, 1]].append((e, 1))
        m["g_ParticleEdgeRanges"], m["g_ParticleIncidentEdges"] = _incidence(N, refs)
        refs = [[] for _ in range(N)]
        for b in range(Bn):
            for slot in range(3):
                refs[m["g_SoftBends"][b, slot]].append((b, slot))
        for d in range(D):
            for slot in range(4):
                refs[m["g_ClothDihedrals"][d, slot]].append((Bn + d, slot))
        m["g_ParticleBendRanges"], m["g_ParticleIncidentBends"] = _incidence(N, refs)
        refs = [[] for _ in range(N)]
        for t in range(T):
            for slot in range(4):
                refs[tets[t, slot]].append((t, slot))
        m["g_ParticleTetRanges"], m["g_ParticleIncidentTets"] = _incidence(N, refs)
        refs = [[] for _ in range(N)]
        for s_ in range(S):
            refs[m["g_StrandSegments"][s_, 0]].append((s_, 0))
            refs[m["g_StrandSegments"][s_, 1]].append((s_, 1))
        m["g_ParticleStrandSegmentRanges"], m["g_ParticleIncidentStrandSegments"] = _incidence(N, refs)
        refs = [[] for _ in range(max(S, 1))]
        for j in range(J):
            refs[m["g_StrandJoints"][j, 0]].append((j, 0))
            refs[m["g_StrandJoints"][j, 1]].append((j, 1))
        m["g_SegmentStrandJointRanges"], m["g_SegmentIncidentStrandJoints"] = _incidence(max(S, 1), refs)

        # rigid bodies and colliders
        B, Cc = soa.rigid_body_count, soa.collider_count
        self.B, self.C = B, Cc
        b1 = max(B, 1)
        m["g_RigidBodyPositionsInvMass"] = _view(soa.body_positions_inv_mass, b1, np.float32, 4) if B else np.zeros((1, 4), np.float32)
        m["g_RigidBodyOrientations"] = _view(soa.body_orientations, b1, np.float32, 4) if B else np.zeros((1, 4), np.float32)
        m["g_RigidBodyLinearVelocities"] = _view(soa.body_linear_velocities, b1, np.float32, 4) if B else np.zeros((1, 4), np.float32)
        m["g_RigidBodyAngularVelocities"] = _view(soa.body_angular_velocities, b1, np.float32, 4) if B else np.zeros((1, 4), np.float32)
        m["g_RigidBodyScales"] = _view(soa.body_scales, b1, np.float32, 4) if B else np.zeros((1, 4), np.float32)
        m["g_RigidBodyInverseInertiaLocal"] = _view(soa.body_inverse_inertia, b1, np.float32, 4) if B else np.zeros((1, 4), np.float32)
        m["g_RigidBodyTypes"] = _view(soa.body_types, b1, np.uint32) if B else np.zeros(1, np.uint32)
        m["g_RigidBodyKinematicTargetPositions"] = _view(soa.body_kinematic_target_positions, b1, np.float32, 4) if B else np.zeros((1, 4), np.float32)
        m["g_RigidBodyKinematicTargetOrientations"] = _view(soa.body_kinematic_target_orientations, b1, np.float32, 4) if B else np.zeros((1, 4), np.float32)
        m["g_RigidBodyKinematicTargetFlags"] = _view(soa.body_kinematic_target_flags, b1, np.uint32) if B else np.zeros(1, np.uint32)
        if B and np.any(m["g_RigidBodyTypes"][:B] == BODY_DYNAMIC):
            raise NotImplementedError("dynamic rigid bodies are not driven by this host pipeline")
        for pre in ("Previous", "Predicted"):
            m[f"g_{pre}RigidBodyPositionsInvMass"] = m["g_RigidBodyPositionsInvMass"].copy()
            m[f"g_{pre}RigidBodyOrientations"] = m["g_RigidBodyOrientations"].copy()
        m["g_PredictedRigidBodyLinearVelocities"] = m["g_RigidBodyLinearVelocities"].copy()
        m["g_PredictedRigidBodyAngularVelocities"] = m["g_RigidBodyAngularVelocities"].copy()
        for k in ("Translation", "Rotation", "LinearVelocity", "AngularVelocity"):
            m[f"g_RigidBody{k}Corrections"] = np.zeros((b1, 4), np.uint32)
        m["g_BodyColliderRanges"] = _view(soa.body_collider_ranges, b1, np.uint32, 2) if B else np.zeros((1, 2), np.uint32)
        m["g_BodyColliderIndices"] = _view(soa.body_collider_indices, max(soa.body_collider_index_count, 1), np.uint32)
        c1 = max(Cc, 1)
        m["g_ColliderGeometryData"] = _records(soa.collider_geometry, c1, 48) if Cc else np.zeros((1, 12), np.uint32)
        m["g_ColliderBroadPhaseData"] = _records(soa.collider_broadphase, c1, 32) if Cc else np.zeros((1, 8), np.uint32)
        m["g_ColliderMaterials"] = _view(soa.collider_materials, c1, np.float32, 4) if Cc else np.zeros((1, 4), np.float32)
        bp = m["g_ColliderBroadPhaseData"]
        m["g_ColliderOwnerRigidBodyIndices"] = np.ascontiguousarray(bp[:, 0])
        m["g_ColliderShapeTypes"] = np.ascontiguousarray(bp[:, 1])
        m["g_ColliderEnabledFlags"] = np.ascontiguousarray(bp[:, 5])
        m["g_BodyAabbs"] = np.zeros((c1, 8), np.float32)
        m["g_BodyMeta"] = np.zeros((c1, 4), np.uint32)
        m["g_ActiveBodyFlags"] = np.zeros(c1, np.uint32)
        m["g_StaticBodyFlags"] = np.zeros(c1, np.uint32)
        m["g_BvhNodes"] = np.zeros((2 * c1, 10), np.uint32)
        m["g_StaticBvhNodes"] = np.zeros((2 * c1, 10), np.uint32)
        m["g_BroadPhaseMeta"] = np.zeros(8, np.uint32)

        # transient particle buffers
        self.cellCap = _next_pow2(max(N * 2, 1))
        self.pairCap = max(N * pair_capacity_per_particle, 1)
        self.maxNb = int(desc.max_fluid_neighborhood) or 128
        m["g_FluidIterationDelta"] = np.zeros((N, 4), np.float32)
        m["g_FluidDeltaPositions"] = np.zeros((N, 4), np.float32)
        m["g_FluidSurfaceNormalConstraints"] = np.zeros((N, 4), np.float32)
        m["g_FluidVorticities"] = np.zeros((N, 4), np.float32)
        m["g_FluidNeighborPairs"] = np.zeros((max(N * self.maxNb, 1), 4), np.uint32)
        m["g_ParticleBroadPhaseEntries"] = np.zeros((max(N, 1), 8), np.uint32)
        m["g_ParticleBroadPhaseKeys"] = np.zeros((max(N, 1), 2), np.uint32)
        m["g_ParticleCellRanges"] = np.zeros((self.cellCap, 4), np.uint32)
        scan = max(N, self.pairCap, 1)
        m["radixFlags"] = np.zeros(scan, np.uint32)
        m["radixOffsets"] = np.zeros(scan, np.uint32)
        m["fbCounts"] = np.zeros(max(N, 1), np.uint32)
        m["fbOffsets"] = np.zeros(max(N, 1), np.uint32)
        m["g_FluidBoundaryCandidateRanges"] = np.zeros((max(N, 1), 2), np.uint32)
        m["g_FluidBoundaryCandidatePairs"] = np.zeros((self.pairCap, 4), np.uint32)
        m["g_ParticleNeighborMeta"] = np.zeros(13, np.uint32)
        m["softRigidPairs"] = np.zeros((self.pairCap, 4), np.uint32)
        m["softSoftPairs"] = np.zeros((self.pairCap, 4), np.uint32)
        m["softRigidContacts"] = np.zeros((self.pairCap, 16), np.uint32)
        m["activeSoftRigidContacts"] = np.zeros((self.pairCap, 16), np.uint32)
        m["softContacts"] = np.zeros((self.pairCap, 12), np.uint32)
        m["activeSoftContacts"] = np.zeros((self.pairCap, 12), np.uint32)
        m["g_ParticlePositionCorrections"] = np.zeros((max(N, 1), 4), np.uint32)
        m["g_ParticleVelocityCorrections"] = np.zeros((max(N, 1), 4), np.uint32)
        # names that bind the same buffer in every pass
        m["g_SortedParticleBroadPhaseKeys"] = m["g_ParticleBroadPhaseKeys"]
        m["g_ParticleVelocitiesRW"] = m["g_ParticleVelocities"]
        m["g_FluidIterationDeltaRW"] = m["g_FluidIterationDelta"]
        self.m = m
        self.cell_size = float(soa.particle_grid_cell_size)
        self.fluid_count = int(np.count_nonzero(m["g_ParticleKinds"] == KIND_FLUID))
        self.nb_counts = None

    # ------------------------------------------------------------------ constants
    def _iterations(self):
        d = self.desc
        base = max(int(d.default_iterations), 1)
        res = lambda v: int(v) if int(v) > 0 else base
        return dict(fluid=res(d.fluid_iterations), soft=res(d.soft_internal_iterations),
                    contact=res(d.soft_contact_iterations), joint=res(d.rigid_joint_iterations),
                    rr=res(d.rigid_rigid_contact_iterations))

    def _config(self):
        """GpuPhysicsSolverConfig (physics_solver.cpp:100-129): the five settings structs."""
        d = self.desc
        vals = []
        for part in (d.contact, d.rigid, d.joints, d.soft, d.fluid):
            vals += list(np.frombuffer(bytes(part), np.float32))
        v = np.array(vals, np.float32).reshape(10, 4)
        names = ["g_ContactSolverConfig0", "g_ContactSolverConfig1", "g_RigidSolverConfig0", "g_RigidSolverConfig1",
                 "g_JointSolverConfig0", "g_JointSolverConfig1", "g_SoftSolverConfig0", "g_SoftSolverConfig1",
                 "g_FluidSolverConfig0", "g_FluidSolverConfig1"]
        return {n: v[i] for i, n in enumerate(names)}

    def run(self, kernel, threads, consts, alias=None):
        self.L[kernel].run(self.m, consts, threads, alias)

    # ------------------------------------------------------------------ helper steps
    def _scan(self, counts_key, offsets_key, n):
        c = self.m[counts_key][:n].astype(np.uint64)
        off = np.zeros(n, np.uint64)
        if n > 1:
            off[1:] = np.cumsum(c[:-1])
        self.m[offsets_key][:n] = off.astype(np.uint32)

    def _meta(self, field):
        names = ["pp", "pr", "fb", "req_pp", "req_pr", "req_fb", "ov_pp", "ov_pr", "ov_fb", "active_pc", "active_prc"]
        return int(self.m["g_ParticleNeighborMeta"][names.index(field)])

    def _build_bvh(self):
        """Chain BVHs over the moving and the static colliders' world AABBs (see the module
        docstring), and GpuBroadPhaseMeta's moving / static counts."""
        m = self.m
        moving = [c for c in range(self.C) if m["g_ActiveBodyFlags"][c]]
        static = [c for c in range(self.C) if m["g_StaticBodyFlags"][c]]
        for key, cols in (("g_BvhNodes", moving), ("g_StaticBvhNodes", static)):
            nodes = m[key]
            nodes[:] = 0
            if not cols:
                continue
            k = len(cols)
            boxes = m["g_BodyAabbs"]

            def leaf(slot, c):
                nodes[slot, 0] = np.uint32(0xFFFFFFFF)
                nodes[slot, 1] = np.uint32(0xFFFFFFFF)
                nodes[slot, 2] = c
                nodes[slot, 3:6] = boxes[c, 0:3].view(np.uint32)
                nodes[slot, 6:9] = boxes[c, 4:7].view(np.uint32)

            if k == 1:
                leaf(0, cols[0])
                continue
            # internal node i (0..k-2): right = leaf of cols[i], left = internal i+1 (the last
            # internal node's left is the leaf of cols[k-1]); leaves at k-1+i.
            for i, c in enumerate(cols):
                leaf(k - 1 + i, c)
            for i in range(k - 2, -1, -1):
                right = k - 1 + i
                left = i + 1 if i < k - 2 else k - 1 + (k - 1)
                nodes[i, 0] = left
                nodes[i, 1] = right
                nodes[i, 2] = 0xFFFFFFFF
                lo = np.minimum(nodes[left, 3:6].view(np.float32), nodes[right, 3:6].view(np.float32))
                hi = np.maximum(nodes[left, 6:9].view(np.float32), nodes[right, 6:9].view(np.float32))
                nodes[i, 3:6] = lo.view(np.uint32)
                nodes[i, 6:9] = hi.view(np.uint32)
        m["g_BroadPhaseMeta"][0] = len(moving)
        m["g_BroadPhaseMeta"][1] = len(static)
        m["g_BroadPhaseMeta"][5] = 1 if static else 0

    def _candidates(self, kind, pc, alias_pairs):
        """count -> scan -> finalize -> emit (physics_pass_dispatcher.cpp candidate builders)."""
        N = self.N
        if kind == "fluid_boundary":
            counts, offs = "fbCounts", "fbOffsets"
            a = {"g_CandidateCounts": counts, "g_CandidateOffsets": offs,
                 "g_CandidateRanges": "g_FluidBoundaryCandidateRanges",
                 "g_ParticleCandidatePairs": "g_FluidBoundaryCandidatePairs"}
        else:
            counts, offs = "radixFlags", "radixOffsets"
            a = {"g_CandidateCounts": counts, "g_CandidateOffsets": offs, "g_ParticleCandidatePairs": alias_pairs}
        self.run(f"particle_count_{kind}_candidates", N, pc, a)
        self._scan(counts, offs, N)
        self.run(f"particle_finalize_{kind}_candidates", 1, pc, a)
        self.run(f"particle_emit_{kind}_candidates", N, pc, a)

    # ------------------------------------------------------------------ one frame
    def step(self, frame_dt: float):
        d = self.desc
        m = self.m
        N, B, Cc = self.N, self.B, self.C
        it = self._iterations()
        substeps = max(int(d.substeps), 1)
        dt = np.float32(frame_dt) / np.float32(substeps)
        max_it = max(it.values())
        cfg = self._config()
        g = np.array([d.gravity[0], d.gravity[1], d.gravity[2], 0.0], np.float32)
        c = self.counts
        for _sub in range(substeps):
            # physics_solver.cpp:437-471
            rc = dict(gravity=g, dt=float(dt), rigidBodyCount=B, colliderCount=Cc,
                      candidatePairCapacity=self.pairCap, contactCapacity=self.pairCap, **cfg)
            pc = dict(dt=float(dt), gravity=g, particleCount=N, rigidColliderCount=Cc,
                      particleGridCellSize=self.cell_size, particleCandidatePairCapacity=self.pairCap,
                      fluidBoundaryCandidatePairCapacity=self.pairCap, maxFluidNeighborhood=self.maxNb,
                      particleCellRangeCapacity=self.cellCap, softEdgeCount=c["E"], softBendCount=c["Bn"],
                      clothDihedralCount=c["D"], softTetCount=c["T"], strandSegmentCount=c["S"],
                      strandJointCount=c["J"], strandDistanceCount=c["Ds"], fluidIterations=it["fluid"],
                      iterationIndex=0, **cfg)
            has_fluid = self.fluid_count > 0 and N > 0
            has_soft = N > 0 and any(c[k] for k in ("E", "Bn", "D", "T", "S", "J", "Ds"))
            has_ss = it["contact"] > 0 and N > 1
            has_rc = N > 0 and Cc > 0
            has_sr = it["contact"] > 0 and has_rc
            has_bp = has_ss or has_fluid or has_rc
            # physics_solver.cpp:497-600
            if B:
                self.run("rigid_clear_corrections", B, rc)
                self.run("rigid_predict", B, rc)
                self.run("rigid_update_world_aabbs", Cc, rc)
                if Cc:
                    self._build_bvh()
                rc["activeMovingCount"] = int(m["g_BroadPhaseMeta"][0])
                rc["staticBodyCount"] = int(m["g_BroadPhaseMeta"][1])
            self.run("soft_predict", N, pc)
            if N and B:
                self.run("particle_sync_rigid_proxy_particles", N, pc)
            if has_bp:
                self.run("particle_build_broad_phase_entries", N, pc)
                self.run("particle_build_broad_phase_keys", N, pc)
                keys = m["g_ParticleBroadPhaseKeys"][:N]
                order = np.argsort(keys[:, 0], kind="stable")
                keys[:] = keys[order]
                self.run("particle_clear_cell_ranges", self.cellCap, pc)
                a = {"g_SortedParticleBroadPhaseKeys": "g_ParticleBroadPhaseKeys",
                     "g_ParticleCellRangeStartFlags": "radixFlags", "g_ParticleCellRangeStartOffsets": "radixOffsets"}
                self.run("particle_mark_cell_range_starts", N, pc, a)
                self._scan("radixFlags", "radixOffsets", N)
                self.run("particle_build_cell_ranges", N, pc, a)
            m["g_ParticleNeighborMeta"][:] = 0
            if N:
                if has_ss:
                    self._candidates("particle_particle", pc, "softSoftPairs")
                if has_rc:
                    self._candidates("particle_rigid", pc, "softRigidPairs")
                if has_fluid and Cc:
                    self._candidates("fluid_boundary", pc, None)
            # physics_clear_soft_constraint_state (physics_solver.cpp:722-735)
            threads = max(N, c["E"], c["Bn"] + c["D"], c["T"], c["S"], c["J"], c["Ds"])
            if has_soft or has_ss or has_sr:
                self.run("clear_soft_constraint_state", threads, pc)
            for itx in range(max_it):
                pc["iterationIndex"] = itx
                run_soft = has_soft and itx < it["soft"]
                run_ss = has_ss and itx < it["contact"]
                run_sr = has_sr and itx < it["contact"]
                run_fluid = has_fluid and itx < it["fluid"]
                if run_fluid:
                    self._fluid_neighbors(pc)
                    fa = {"g_FluidNeighborCounts": "radixFlags"}
                    self.run("fluid_compute_density_lambda", N, pc, fa)
                    self.run("fluid_compute_delta_positions", N, pc, fa)
                    self.run("fluid_apply_delta_positions", N, pc)
                    self.run("fluid_clamp_boundary", N, pc, {"g_FluidIterationDeltaRW": "g_FluidIterationDelta"})
                if run_soft:
                    self.run("soft_solve_edge_constraints", c["E"], pc)
                    self.run("soft_apply_edge_corrections", N, pc)
                    self.run("strand_solve_segment_constraints", c["S"], pc)
                    self.run("strand_apply_segment_corrections", max(N, c["S"]), pc)
                    self.run("soft_solve_bend_constraints", c["Bn"], pc)
                    self.run("cloth_solve_dihedral_constraints", c["D"], pc)
                    self.run("soft_apply_bend_corrections", N, pc)
                    self.run("strand_solve_joint_constraints", c["J"], pc)
                    self.run("strand_apply_joint_corrections", c["S"], pc)
                    self.run("strand_solve_distance_constraints", c["Ds"], pc)
                    self.run("strand_apply_distance_corrections", N, pc)
                    self.run("soft_solve_tet_constraints", c["T"], pc)
                    self.run("soft_apply_tet_corrections", N, pc)
                if run_ss:
                    a = {"g_ParticleCandidatePairs": "softSoftPairs", "g_ContactActiveFlags": "radixFlags",
                         "g_ContactActiveOffsets": "radixOffsets", "g_ParticleContacts": "softContacts",
                         "g_ActiveSoftContacts": "activeSoftContacts"}
                    n = self._meta("pp")
                    self.run("particle_generate_explicit_contacts", n, pc, a)
                    self._scan("radixFlags", "radixOffsets", n)
                    self.run("particle_finalize_active_explicit_contacts", 1, pc, a)
                    self.run("particle_compact_active_explicit_contacts", n, pc, a)
                if run_sr:
                    a = {"g_ParticleCandidatePairs": "softRigidPairs", "g_ContactActiveFlags": "radixFlags",
                         "g_ContactActiveOffsets": "radixOffsets", "g_ParticleRigidContacts": "softRigidContacts",
                         "g_ActiveSoftRigidContacts": "activeSoftRigidContacts"}
                    n = self._meta("pr")
                    self.run("particle_rigid_generate_contacts", n, pc, a)
                    self._scan("radixFlags", "radixOffsets", n)
                    self.run("particle_finalize_active_rigid_contacts", 1, pc, a)
                    self.run("particle_compact_active_rigid_contacts", n, pc, a)
                if run_ss:
                    prev = {"g_PreviousRigidBodyPositionsInvMass": "g_RigidBodyPositionsInvMass",
                            "g_PreviousRigidBodyOrientations": "g_RigidBodyOrientations",
                            "g_ParticleContacts": "activeSoftContacts"}
                    self.run("particle_solve_explicit_contacts", self._meta("active_pc"), {**pc, **rc}, prev)
                if run_sr:
                    prev = {"g_PreviousRigidBodyPositionsInvMass": "g_RigidBodyPositionsInvMass",
                            "g_PreviousRigidBodyOrientations": "g_RigidBodyOrientations",
                            "g_ParticleRigidContacts": "activeSoftRigidContacts"}
                    self.run("particle_rigid_solve_contacts", self._meta("active_prc"), {**pc, **rc}, prev)
                if run_ss or run_sr:
                    self.run("particle_apply_position_corrections", N, pc)
                if run_sr and B:
                    self.run("rigid_apply_corrections", B, rc)
                    if N:
                        self.run("particle_sync_rigid_proxy_particles", N, pc)
            # physics_solver.cpp:1241-1300
            if B:
                self.run("rigid_update_velocities", B, rc)
            self.run("particle_update_velocities", N, pc)
            if has_fluid:
                self.run("fluid_project_boundary_velocities", N, pc)
                # post-update neighbour rebuild and vorticity confinement (physics_solver.cpp:1262-1285)
                self._fluid_neighbors(pc)
                va = {"g_FluidNeighborCounts": "radixFlags", "g_ParticleVelocitiesRW": "g_ParticleVelocities"}
                self.run("fluid_compute_vorticity", N, pc, va)
                self.run("fluid_apply_vorticity_confinement", N, pc, va)
            if has_ss and it["contact"] > 0:
                a = {"g_ParticleContacts": "activeSoftContacts"}
                for _ in range(it["contact"]):
                    self.run("particle_solve_contact_velocities", self._meta("active_pc"), {**pc, **rc}, a)
                    self.run("particle_apply_contact_velocities", N, pc)
                    if B:
                        self.run("rigid_apply_contact_velocities", B, rc)
            if has_sr and it["contact"] > 0:
                a = {"g_ParticleRigidContacts": "activeSoftRigidContacts"}
                for _ in range(it["contact"]):
                    self.run("particle_rigid_solve_contact_velocities", self._meta("active_prc"), {**pc, **rc}, a)
                    self.run("particle_apply_contact_velocities", N, pc)
                    self.run("rigid_apply_contact_velocities", B, rc)
            # copyPredictedRigidBodiesToPersistentState
            if B:
                m["g_RigidBodyPositionsInvMass"][:] = m["g_PredictedRigidBodyPositionsInvMass"]
                m["g_RigidBodyOrientations"][:] = m["g_PredictedRigidBodyOrientations"]
                m["g_RigidBodyLinearVelocities"][:] = m["g_PredictedRigidBodyLinearVelocities"]
                m["g_RigidBodyAngularVelocities"][:] = m["g_PredictedRigidBodyAngularVelocities"]
        oor, barriers = self.L.counters()
        if barriers:
            raise RuntimeError("a kernel reached a group barrier")
        return oor

    def _fluid_neighbors(self, pc):
        a = {"g_SortedParticleBroadPhaseKeys": "g_ParticleBroadPhaseKeys", "g_CandidateCounts": "radixFlags"}
        self.run("fluid_build_neighbors", self.N, pc, a)
        self.nb_counts = self.m["radixFlags"][:self.N].copy()

    # ------------------------------------------------------------------ readback
    def set_kinematic_target(self, body, position, orientation=(0, 0, 0, 1)):
        self.m["g_RigidBodyKinematicTargetPositions"][body, :3] = position
        self.m["g_RigidBodyKinematicTargetOrientations"][body] = orientation
        self.m["g_RigidBodyKinematicTargetFlags"][body] = 1

    def read_particles(self):
        return (self.m["g_ParticlePositionsInvMass"].copy(), self.m["g_ParticleVelocities"].copy(),
                self.m["g_ParticlePreviousPositions"].copy())

    def debug_read(self, name: str) -> np.ndarray:
        """The oracle's debug views (cn_oracle.Oracle.debug_read) of the reference's buffers."""
        if name == "sorted_keys":
            return np.ascontiguousarray(self.m["g_ParticleBroadPhaseKeys"][:self.N]).view(np.uint8).ravel()
        if name == "fluid_neighbor_counts":
            # physics_fluid_build_neighbors.cs.hlsl:30-39: particles that are not fluid, or are
            # pinned, leave their entry of the shared count buffer untouched; report 0 for them.
            live = (self.m["g_ParticleKinds"] == KIND_FLUID) & (self.m["g_ParticlePositionsInvMass"][:, 3] > 1e-6)
            return np.ascontiguousarray(np.where(live, self.nb_counts, 0).astype(np.uint32)).view(np.uint8).ravel()
        if name == "fluid_neighbors":
            pairs = self.m["g_FluidNeighborPairs"].reshape(self.N, self.maxNb, 4)
            return np.ascontiguousarray(pairs[:, :, 2]).view(np.uint8).ravel()
        raise KeyError(name)

    def neighbor_lists(self):
        """Per particle, the neighbour indices of the last build, in slot order."""
        pairs = self.m["g_FluidNeighborPairs"].reshape(self.N, self.maxNb, 4)
        return [pairs[i, :self.nb_counts[i], 2].copy() for i in range(self.N)]
