"""The C-ABI library loads and exports every entry point include/cn_physics.h declares (no GPU)."""
import ctypes as C
import re
from pathlib import Path

import pytest

from cn_physics import _abi, load, solver_desc
from conftest import has_gpu

HEADER = Path(__file__).resolve().parent.parent / "include" / "cn_physics.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"CN_API\s+[\w\s\*]+?\b(cn_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "cn_solver_step" in syms and "cn_world_get_soa" in syms and len(syms) >= 30


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(_abi.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_mirror_binds_every_declared_symbol():
    bound = {name for name, _, _ in _abi.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_struct_sizes_match_header():
    import subprocess, tempfile, os
    src = r'''
#include <stdio.h>
#include "cn_physics.h"
int main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n",
 sizeof(cn_solver_desc),
 sizeof(cn_world_soa), sizeof(cn_soft_body_grid_desc), sizeof(cn_fluid_grid_desc), sizeof(cn_cloth_grid_desc),
 sizeof(cn_strand_desc), sizeof(cn_rigid_body_desc), sizeof(cn_collider_desc), sizeof(cn_meta), sizeof(cn_scene_view),
 sizeof(cn_batch_desc), sizeof(cn_batch_stats), sizeof(cn_batch_tuning), sizeof(cn_server_desc),
 sizeof(cn_request_done), sizeof(cn_server_stats), sizeof(cn_diff_desc), sizeof(cn_surface_vertex_binding),
 sizeof(cn_surface_triangle_range), sizeof(cn_surface_render_data), sizeof(cn_surface_mesh_desc),
 sizeof(cn_surface_render_view), sizeof(cn_rigid_proxy_desc), sizeof(cn_schedule_info), sizeof(cn_soft_settings)); return 0;}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "s.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "s")
        cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
        subprocess.run([cc, "-I", str(HEADER.parent), c, "-o", exe], check=True)
        got = list(map(int, subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()))
    want = [C.sizeof(t) for t in (_abi.SolverDesc, _abi.WorldSoA, _abi.SoftBodyGridDesc, _abi.FluidGridDesc,
                                  _abi.ClothGridDesc, _abi.StrandDesc, _abi.RigidBodyDesc, _abi.ColliderDesc,
                                  _abi.Meta, _abi.SceneView, _abi.BatchDesc, _abi.BatchStats, _abi.BatchTuning,
                                  _abi.ServerDesc, _abi.RequestDone, _abi.ServerStats, _abi.DiffDesc,
                                  _abi.SurfaceVertexBinding, _abi.SurfaceTriangleRange, _abi.SurfaceRenderData,
                                  _abi.SurfaceMeshDesc, _abi.SurfaceRenderView, _abi.RigidProxyDesc,
                                  _abi.ScheduleInfo, _abi.SoftSettings)]
    assert got == want


def test_record_layouts_are_reference_sized():
    # physics_particle_types.hlsli:111-290 record sizes
    assert C.sizeof(_abi.FluidMaterial) == 48
    # SurfaceRenderVertexBinding / SurfaceRenderVertexTriangleRange (physics_types.h:1350-1363)
    assert C.sizeof(_abi.SurfaceVertexBinding) == 32 and C.sizeof(_abi.SurfaceTriangleRange) == 16


def test_defaults_mirror_reference_desc():
    d = solver_desc()
    assert d.default_iterations == 20 and d.substeps == 1 and abs(d.gravity[1] + 9.81) < 1e-6
    assert abs(d.soft.internal_relaxation - 0.2) < 1e-7
    assert abs(d.contact.slop - 1e-3) < 1e-9 and abs(d.contact.soft_relaxation - 0.95) < 1e-7
    assert abs(d.fluid.constraint_relaxation - 0.7) < 1e-7 and abs(d.fluid.boundary_density_scale - 0.12) < 1e-7
    assert d.enable_blocking_readback == 1 and d.max_fluid_neighborhood == 128


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_solver_create_fails_loudly_without_device():
    lib = load()
    h = C.c_void_p()
    d = solver_desc()
    status = lib.cn_solver_create(C.byref(d), 0, C.byref(h))
    assert status == 6  # CN_ERR_NO_DEVICE: there is no CPU fallback
    assert b"no CUDA device" in lib.cn_last_error()
