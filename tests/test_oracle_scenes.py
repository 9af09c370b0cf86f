"""The numpy restatement of the dam break that bench.py's reference arm builds for the oracle
(oracle/cn_scenes.py, so that arm loads no product library) equals the product World's SoA byte
for byte, and its solver defaults equal cn_solver_desc_defaults."""
import ctypes as C

import numpy as np

import cn_scenes
from cn_physics import _abi, load, scenes


def _arr(ptr, nbytes):
    if nbytes == 0:
        return b""
    return bytes((C.c_uint8 * nbytes).from_address(C.cast(ptr, C.c_void_p).value))


def test_reference_desc_equals_the_library_defaults():
    d = _abi.SolverDesc()
    load().cn_solver_desc_defaults(C.byref(d))
    assert bytes(cn_scenes.reference_desc()) == bytes(d)


def test_dam_break_soa_equals_the_world_soa():
    dims = (16, 12, 20)
    ref = cn_scenes.DamBreak(*dims, box=(1.6, 1.2, 2.4))
    w, desc, dt = scenes.dam_break(*dims, box=(1.6, 1.2, 2.4))
    a, b = ref.soa(), w.soa()
    n = b.particle_count
    assert a.particle_count == n
    assert bytes(ref.desc) == bytes(desc) and ref.frame_dt == dt
    for field, size in (("positions_inv_mass", 16 * n), ("velocities", 16 * n), ("radii", 4 * n), ("kinds", 4 * n),
                        ("metadata", 16 * n), ("material_indices", 4 * n), ("fluid_material_indices", 4 * n),
                        ("owner_types", 4 * n), ("owner_indices", 4 * n), ("adjacency_offsets", 4 * n),
                        ("adjacency_counts", 4 * n), ("contact_materials", 16 * b.contact_material_count),
                        ("fluid_materials", 48 * b.fluid_material_count), ("collider_geometry", 48 * b.collider_count),
                        ("collider_broadphase", 32 * b.collider_count), ("collider_materials", 16 * b.collider_count),
                        ("body_positions_inv_mass", 16), ("body_orientations", 16), ("body_scales", 16),
                        ("body_types", 4), ("body_collider_ranges", 8), ("body_collider_indices", 20)):
        assert _arr(getattr(a, field), size) == _arr(getattr(b, field), size), field
    for field in ("contact_material_count", "fluid_material_count", "adjacency_index_count", "rigid_body_count",
                  "collider_count", "body_collider_index_count", "edge_count", "tet_count"):
        assert getattr(a, field) == getattr(b, field), field
    assert np.float32(a.particle_grid_cell_size) == np.float32(b.particle_grid_cell_size)
