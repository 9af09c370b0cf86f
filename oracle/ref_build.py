"""Build recipe: the reference's own HLSL compute shaders, compiled for the host CPU.

TEST INFRASTRUCTURE ONLY.  The reference (CRESSim-Neo) runs its physics substep as HLSL compute
shaders through Diligent Engine and DXC, which cannot be built here.  The shaders themselves are
plain compute code, so this recipe compiles them with g++ against the project-written HLSL model
in oracle/hlsl_host.h and executes them one thread at a time (oracle/ref_kernels.py):

  1. the C preprocessor expands each shader with the reference's include directories
     (assets/shaders/include/**), exactly as DXC would see it;
  2. the few HLSL constructs C++ cannot parse are rewritten: [numthreads]/[loop]/... attributes
     and SV_ semantics removed, cbuffer blocks opened into globals, out/inout parameters made
     references, swizzles such as .xyz made calls into hlsl_host.h, float literals given the
     float type (HLSL literals take the type of the float operand they meet), (T)0 made T{};
  3. the result is wrapped in a namespace per shader with a generated binding table (buffers,
     constants, numthreads, a dispatch loop over SV_DispatchThreadID) and compiled with
     -ffp-contract=off into oracle/_ref/libcn_ref_shaders.so.

The shader sources are read in place under the reference tree and are not copied anywhere: the
rewritten translation unit reaches g++ through a pipe, and only objects and the shared library
are written, to oracle/_ref/ (git-ignored).  Kernels that synchronise a thread group (GroupMemoryBarrierWithGroupSync: the block
scan, the rigid extent reductions) are not built; the host driver computes those steps directly.

Usage: python oracle/ref_build.py [--reference /root/reference] [--force]
"""
from __future__ import annotations

import hashlib
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
LIB = OUT / "libcn_ref_shaders.so"
DEFAULT_REFERENCE = Path(os.environ.get("CN_REFERENCE_ROOT", "/root/reference"))

# Hot-path shaders of PhysicsSolver::step (src/physics/physics_solver.cpp:336-1401) that run one
# thread at a time without group barriers.
SHADERS = [
    "physics/soft/solver/physics_soft_predict.cs.hlsl",
    "physics/particle/solver/physics_particle_update_velocities.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_build_broad_phase_entries.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_build_broad_phase_keys.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_mark_cell_range_starts.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_clear_cell_ranges.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_build_cell_ranges.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_count_fluid_boundary_candidates.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_finalize_fluid_boundary_candidates.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_emit_fluid_boundary_candidates.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_count_particle_particle_candidates.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_finalize_particle_particle_candidates.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_emit_particle_particle_candidates.cs.hlsl",
    "physics/particle/narrow_phase/physics_particle_generate_explicit_contacts.cs.hlsl",
    "physics/particle/narrow_phase/physics_particle_compact_active_explicit_contacts.cs.hlsl",
    "physics/particle/narrow_phase/physics_particle_finalize_active_explicit_contacts.cs.hlsl",
    "physics/particle/narrow_phase/physics_particle_finalize_active_rigid_contacts.cs.hlsl",
    "physics/particle/solver/physics_particle_solve_explicit_contacts.cs.hlsl",
    "physics/particle/solver/physics_particle_solve_contact_velocities.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_count_particle_rigid_candidates.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_finalize_particle_rigid_candidates.cs.hlsl",
    "physics/particle/broad_phase/physics_particle_emit_particle_rigid_candidates.cs.hlsl",
    "physics/particle/narrow_phase/physics_particle_rigid_generate_contacts.cs.hlsl",
    "physics/particle/narrow_phase/physics_particle_compact_active_rigid_contacts.cs.hlsl",
    "physics/particle/solver/physics_particle_rigid_solve_contacts.cs.hlsl",
    "physics/particle/solver/physics_particle_apply_position_corrections.cs.hlsl",
    "physics/particle/solver/physics_particle_rigid_solve_contact_velocities.cs.hlsl",
    "physics/particle/solver/physics_particle_apply_contact_velocities.cs.hlsl",
    "physics/fluid/solver/physics_fluid_build_neighbors.cs.hlsl",
    "physics/fluid/solver/physics_fluid_compute_density_lambda.cs.hlsl",
    "physics/fluid/solver/physics_fluid_compute_delta_positions.cs.hlsl",
    "physics/fluid/solver/physics_fluid_apply_delta_positions.cs.hlsl",
    "physics/fluid/solver/physics_fluid_clamp_boundary.cs.hlsl",
    "physics/fluid/solver/physics_fluid_project_boundary_velocities.cs.hlsl",
    "physics/fluid/solver/physics_fluid_compute_vorticity.cs.hlsl",
    "physics/fluid/solver/physics_fluid_apply_vorticity_confinement.cs.hlsl",
    "physics/shared/physics_clear_soft_constraint_state.cs.hlsl",
    "physics/soft/solver/physics_soft_solve_edge_constraints.cs.hlsl",
    "physics/soft/solver/physics_soft_apply_edge_corrections.cs.hlsl",
    "physics/soft/solver/physics_soft_solve_tet_constraints.cs.hlsl",
    "physics/soft/solver/physics_soft_apply_tet_corrections.cs.hlsl",
    "physics/soft/solver/physics_soft_solve_bend_constraints.cs.hlsl",
    "physics/soft/solver/physics_cloth_solve_dihedral_constraints.cs.hlsl",
    "physics/soft/solver/physics_soft_apply_bend_corrections.cs.hlsl",
    "physics/soft/solver/physics_strand_solve_segment_constraints.cs.hlsl",
    "physics/soft/solver/physics_strand_apply_segment_corrections.cs.hlsl",
    "physics/soft/solver/physics_strand_solve_joint_constraints.cs.hlsl",
    "physics/soft/solver/physics_strand_apply_joint_corrections.cs.hlsl",
    "physics/soft/solver/physics_strand_solve_distance_constraints.cs.hlsl",
    "physics/soft/solver/physics_strand_apply_distance_corrections.cs.hlsl",
    "physics/rigid/solver/physics_rigid_predict.cs.hlsl",
    "physics/rigid/broad_phase/physics_rigid_update_world_aabbs.cs.hlsl",
    "physics/rigid/solver/physics_rigid_clear_corrections.cs.hlsl",
    "physics/rigid/solver/physics_rigid_apply_corrections.cs.hlsl",
    "physics/rigid/solver/physics_rigid_apply_contact_velocities.cs.hlsl",
    "physics/rigid/solver/physics_rigid_update_velocities.cs.hlsl",
    "physics/particle/solver/physics_particle_sync_rigid_proxy_particles.cs.hlsl",
]

ATTR_RE = re.compile(r"\[\s*(numthreads|loop|unroll|branch|flatten|fastopt|allow_uav_condition|call|earlydepthstencil)"
                     r"\s*(\([^\]]*\))?\s*\]")
SEMANTIC_RE = re.compile(r":\s*(SV_\w+|register\s*\([^)]*\)|packoffset\s*\([^)]*\))")
CBUFFER_RE = re.compile(r"\bcbuffer\s+(\w+)\s*\{")
PARAM_QUAL_RE = re.compile(r"\b(inout|out)\s+((?:const\s+)?[A-Za-z_][\w:]*(?:<[^<>]*>)?)\s+([A-Za-z_]\w*)"
                            r"(\s*\[\s*\w+\s*\])?")
IN_QUAL_RE = re.compile(r"([(,]\s*)in\s+(?=[A-Za-z_])")
ZERO_CAST_RE = re.compile(r"\(\s*([A-Za-z_]\w*)\s*\)\s*0(?![\w.])")
SWIZZLES = "xyz|xy|yz|zw|xz|yx|yyy|zzz|yzx|zxy|yzw"
# .xxx also applies to scalars in HLSL: an identifier or a call (one level of nested parentheses)
# followed by .xxx becomes hlsl::splat3(...).
SPLAT_RE = re.compile(r"(\b[A-Za-z_]\w*(?:\((?:[^()]|\([^()]*\))*\))?)\.xxx\b")
SWIZZLE_RE = re.compile(r"\.(" + SWIZZLES + r")\b(?!\s*\()")
FLOAT_LIT_RE = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")
BUFFER_RE = re.compile(r"\b(RW)?StructuredBuffer\s*<\s*([\w:]+)\s*>\s+(\w+)\s*;")
RAW_BUFFER_RE = re.compile(r"\b(RW)?ByteAddressBuffer\s+(\w+)\s*;")
SCALARS = {"float", "uint", "int", "bool", "double"}
FIELD_RE = re.compile(r"\b([A-Za-z_]\w*)\s+([A-Za-z_]\w*)\s*(\[\s*\d+\s*\])?\s*;")
MAIN_RE = re.compile(r"\bvoid\s+main\s*\(([^)]*)\)")


def include_dirs(reference: Path) -> list[Path]:
    root = reference / "assets" / "shaders" / "include"
    dirs = [root] + sorted(p for p in root.rglob("*") if p.is_dir())
    return dirs


def preprocess(reference: Path, shader: Path) -> str:
    cmd = ["g++", "-E", "-P", "-x", "c++", "-undef", "-D__HLSL_VERSION=2021", "-I", str(shader.parent)]
    for d in include_dirs(reference):
        cmd += ["-I", str(d)]
    cmd.append(str(shader))
    return subprocess.run(cmd, check=True, capture_output=True, text=True).stdout


def open_cbuffers(src: str) -> tuple[str, list[tuple[str, str, str]]]:
    fields: list[tuple[str, str, str]] = []
    while True:
        m = CBUFFER_RE.search(src)
        if not m:
            return src, fields
        depth, i = 1, m.end()
        while depth:
            depth += {"{": 1, "}": -1}.get(src[i], 0)
            i += 1
        body = src[m.end():i - 1]
        for f in FIELD_RE.finditer(body):
            fields.append((f.group(1), f.group(2), f.group(3) or ""))
        j = i
        while j < len(src) and src[j] in " \t\n":
            j += 1
        if j < len(src) and src[j] == ";":
            i = j + 1
        src = src[:m.start()] + body + src[i:]


def rewrite(src: str) -> tuple[str, dict]:
    info: dict = {"numthreads": (1, 1, 1), "params": []}
    m = re.search(r"\[\s*numthreads\s*\(\s*(\d+)\s*,\s*(\d+)\s*,\s*(\d+)\s*\)\s*\]", src)
    if m:
        info["numthreads"] = tuple(int(g) for g in m.groups())
    mm = MAIN_RE.search(src)
    if not mm:
        raise RuntimeError("no main() in shader")
    for p in mm.group(1).split(","):
        p = p.strip()
        if not p:
            continue
        sem = re.search(r":\s*(SV_\w+)", p)
        decl = p.split(":")[0].split()
        info["params"].append((decl[-2], decl[-1], sem.group(1) if sem else ""))
    src = ATTR_RE.sub("", src)
    src = SEMANTIC_RE.sub("", src)
    src, info["constants"] = open_cbuffers(src)
    src = re.sub(r"\bgroupshared\b", "static", src)
    src = re.sub(r"\b(globallycoherent|precise|nointerpolation)\b", "", src)
    src = PARAM_QUAL_RE.sub(lambda q: f"{q.group(2)} (&{q.group(3)}){q.group(4).strip()}" if q.group(4)
                            else f"{q.group(2)} &{q.group(3)}", src)
    src = IN_QUAL_RE.sub(r"\1", src)
    src = ZERO_CAST_RE.sub(r"\1{}", src)
    src = SPLAT_RE.sub(r"hlsl::splat3(\1)", src)
    src = SWIZZLE_RE.sub(r".\1()", src)
    src = FLOAT_LIT_RE.sub(lambda x: x.group(1) + "f", src)
    info["buffers"] = [(b.group(3), b.group(2), bool(b.group(1))) for b in BUFFER_RE.finditer(src)]
    info["buffers"] += [(b.group(2), "uint", bool(b.group(1))) for b in RAW_BUFFER_RE.finditer(src)]
    return src, info


def translation_unit(name: str, src: str, info: dict) -> str:
    ns = "ref_" + name

    def q(t: str) -> str:
        return t if t in SCALARS else f"{ns}::{t}"

    out = [f'#include "hlsl_host.h"', f"namespace {ns} {{", "using namespace hlsl;", src, "}", ""]
    out.append(f'extern "C" int {name}_bind(const char *n, void *p, unsigned long long bytes) {{')
    for bname, btype, _rw in info["buffers"]:
        out.append(f'  if (!std::strcmp(n, "{bname}")) {{ if (bytes % sizeof({q(btype)})) return -2; '
                   f'{ns}::{bname}.data = reinterpret_cast<decltype({ns}::{bname}.data)>(p); '
                   f'{ns}::{bname}.count = bytes / sizeof({q(btype)}); return 0; }}')
    out.append("  return -1;\n}")
    out.append(f'extern "C" int {name}_set(const char *n, const void *p, unsigned long long bytes) {{')
    for ctype, cname, arr in info["constants"]:
        out.append(f'  if (!std::strcmp(n, "{cname}")) {{ if (bytes != sizeof({ns}::{cname})) return -2; '
                   f'std::memcpy((void *)&{ns}::{cname}, p, bytes); return 0; }}')
    out.append("  return -1;\n}")
    nx, ny, nz = info["numthreads"]
    args = []
    for ptype, _pname, sem in info["params"]:
        arg = {"SV_DispatchThreadID": "dtid", "SV_GroupThreadID": "gtid", "SV_GroupID": "gid",
               "SV_GroupIndex": "gidx"}[sem]
        if ptype in ("uint", "int") and arg != "gidx":
            arg += ".x"
        args.append(arg)
    out.append(f'extern "C" void {name}_dispatch(unsigned gx, unsigned gy, unsigned gz) {{')
    out.append("  for (unsigned bz = 0; bz < gz; ++bz) for (unsigned by = 0; by < gy; ++by) for (unsigned bx = 0; bx < gx; ++bx)")
    out.append(f"  for (unsigned tz = 0; tz < {nz}u; ++tz) for (unsigned ty = 0; ty < {ny}u; ++ty) for (unsigned tx = 0; tx < {nx}u; ++tx) {{")
    out.append(f"    const hlsl::uint3 gtid(tx, ty, tz), gid(bx, by, bz), dtid(bx * {nx}u + tx, by * {ny}u + ty, bz * {nz}u + tz);")
    out.append(f"    const unsigned gidx = tz * {nx * ny}u + ty * {nx}u + tx; (void)gidx; (void)gtid; (void)gid; (void)dtid;")
    out.append(f"    {ns}::main({', '.join(args)});")
    out.append("  }\n}")
    desc = ";".join([f"numthreads={nx},{ny},{nz}"] +
                    [f"buffer:{b}:{t}:{'rw' if rw else 'ro'}" for b, t, rw in info["buffers"]] +
                    [f"const:{c}:{t}{a}" for t, c, a in info["constants"]])
    out.append(f'extern "C" const char *{name}_info() {{ return "{desc}"; }}')
    out.append(f'extern "C" unsigned long long {name}_sizeof(const char *n) {{')
    for bname, btype, _rw in info["buffers"]:
        out.append(f'  if (!std::strcmp(n, "{bname}")) return sizeof({q(btype)});')
    out.append("  return 0;\n}")
    return "\n".join(out) + "\n"


COMMON_TU = """#include "hlsl_host.h"
namespace hlsl { int g_barrierCalls = 0; uint64_t g_outOfRange = 0; }
extern "C" unsigned long long cnref_out_of_range() { return hlsl::g_outOfRange; }
extern "C" int cnref_barrier_calls() { return hlsl::g_barrierCalls; }
extern "C" void cnref_reset_counters() { hlsl::g_outOfRange = 0; hlsl::g_barrierCalls = 0; }
"""

CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-w"]


def shader_name(rel: str) -> str:
    stem = Path(rel).name.replace(".cs.hlsl", "")
    return stem[len("physics_"):] if stem.startswith("physics_") else stem


def build(reference: Path = DEFAULT_REFERENCE, force: bool = False, jobs: int = 8) -> Path | None:
    shaders_root = reference / "assets" / "shaders"
    if not shaders_root.is_dir():
        return None
    OUT.mkdir(exist_ok=True)
    own = [Path(__file__), HERE / "hlsl_host.h"]
    stamp = hashlib.sha256(b"".join(p.read_bytes() for p in own)).hexdigest()[:16]

    def one(rel: str) -> Path:
        name = shader_name(rel)
        obj = OUT / f"{name}.o"
        mark = OUT / f"{name}.stamp"
        src_path = shaders_root / rel
        text = preprocess(reference, src_path)
        body, info = rewrite(text)
        code = f"// generated from {rel} (build stamp {stamp})\n" + translation_unit(name, body, info)
        digest = hashlib.sha256(code.encode()).hexdigest()
        if not force and obj.exists() and mark.exists() and mark.read_text() == digest:
            return obj
        # The rewritten unit goes to the compiler through a pipe: no copy of the shader is stored.
        r = subprocess.run(["g++", *CXXFLAGS, "-I", str(HERE), "-x", "c++", "-c", "-", "-o", str(obj)],
                           input=code, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"{rel}: g++ failed\n{r.stderr[-6000:]}")
        mark.write_text(digest)
        return obj

    with ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(one, SHADERS))
    common = OUT / "common.cpp"
    common.write_text(COMMON_TU)
    cobj = OUT / "common.o"
    subprocess.run(["g++", *CXXFLAGS, "-I", str(HERE), "-c", str(common), "-o", str(cobj)], check=True)
    subprocess.run(["g++", "-shared", "-o", str(LIB), str(cobj), *map(str, objs)], check=True)
    return LIB


if __name__ == "__main__":
    ref = DEFAULT_REFERENCE
    if "--reference" in sys.argv:
        ref = Path(sys.argv[sys.argv.index("--reference") + 1])
    lib = build(ref, force="--force" in sys.argv)
    print(lib if lib else "reference tree not found: nothing built")
