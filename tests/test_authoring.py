"""Host authoring against the reference's known answers (no GPU)."""
import numpy as np

from cn_physics import World
import cn_oracle


def test_regular_grid_counts_match_reference():
    # tests/physics/physics_soft_body_generation_regular_tet_grid.cpp:11-41
    w = World()
    w.add_soft_body_grid((2.0, 2.0, 2.0), 1.0, position=(1.0, 2.0, 3.0), mass=2.0, radius=0.15,
                         edge_compliance=0.01, volume_compliance=0.02, self_collision=True, layer=0x8, mask=0x25)
    c = w.counts()
    assert c["particles"] == 27 and c["tets"] == 40 and c["edges"] > 0
    x = w.positions()
    assert np.allclose(x[:, 3], 0.5)                       # invMass = 1 / particleMass
    assert np.allclose(x[:, :3].mean(axis=0), (1.0, 2.0, 3.0))
    meta = w.array("metadata")
    assert (meta[:, 1] & 0x80000000).all()                   # self-collision flag packed in the phase
    assert (meta[:, 2] == 0x8).all() and (meta[:, 3] == 0x25).all()


def test_regular_grid_tets_are_valid_and_edges_unique():
    w = World()
    w.add_soft_body_grid((0.9375, 0.9375, 0.9375), 1.0 / 16.0)
    c = w.counts()
    assert c["particles"] == 16 ** 3 and c["tets"] == 15 ** 3 * 5
    tets = w.array("tets")[:, :4]
    x = w.positions()[:, :3]
    p0, p1, p2, p3 = (x[tets[:, k]] for k in range(4))
    vol = np.abs(np.einsum("ij,ij->i", np.cross(p1 - p0, p2 - p0), p3 - p0)) / 6.0
    assert (vol > 1e-8).all()
    e = w.array("edges")[:, :2]
    assert len({(int(a), int(b)) for a, b in e}) == len(e)
    assert (e[:, 0] < e[:, 1]).all()
    # 5-tet split: 3*15*16*16 axis edges + face diagonals + 1 body diagonal per cell... every cell
    # contributes its 6 face diagonals shared with neighbours; just check the count is plausible
    assert 3 * 15 * 16 * 16 < len(e) < 7 * 16 ** 3


def test_cloth_and_strand_counts_match_reference():
    # tests/physics/physics_soft_gpu_scene_upload.cpp:60-151: two triangles -> one dihedral;
    # three strand points -> two segments and one joint.
    w = World()
    w.add_cloth_grid((2, 2), (1.0, 1.0), static_particles=[2, 3], bend_compliance=0.01)
    w.add_strand([(-0.2, 1.5, 0.0), (0.0, 1.7, 0.0), (0.2, 1.5, 0.0)], mass=0.5, radius=0.05,
                 stretch_shear_compliance=0.01, bend_compliance=0.02, twist_compliance=0.03)
    c = w.counts()
    assert c["dihedrals"] == 1 and c["segments"] == 2 and c["joints"] == 1 and c["distances"] == 2
    assert c["edges"] == 5


def test_fluid_lattice_and_material_match_oracle_restatement():
    w = World()
    w.add_fluid_grid((0.8, 0.4, 0.8), 0.05, radius=0.03, viscosity=0.01)
    c = w.counts()
    assert c["particles"] == 16 * 8 * 16
    fm = w.fluid_materials()[0]
    ref = cn_oracle.fluid_material(0.03, viscosity=0.01)
    assert np.array_equal(fm.view(np.uint32), ref.view(np.uint32))
    assert abs(fm[2] - 0.1) < 1e-6          # h = max((2/0.6) r, 2r)


def test_grid_cell_size_is_max_of_diameter_and_support():
    w = World()
    w.add_soft_body_grid((1, 1, 1), 0.25, radius=0.2)
    w.add_fluid_grid((0.4, 0.4, 0.4), 0.05, radius=0.03)
    assert abs(w.soa().particle_grid_cell_size - 0.4) < 1e-7
