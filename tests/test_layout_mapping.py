"""ParticleLayoutMapping export (include/engine/particle_layout_mapping.h:11-68, filled as
Runtime::tryGetPreparedParticleLayoutMapping does, src/engine/runtime.cpp:867-955): owners' slot
ranges in the packing order (soft bodies, cloth, strands, fluids), strand ids and orders,
owning soft bodies, filters, and a revision that changes with a new packing."""
import numpy as np

from cn_physics import World

OWNER_SOFT, OWNER_FLUID, OWNER_STRAND, OWNER_CLOTH = 1, 2, 3, 5


def world():
    w = World()
    w.add_soft_body_grid((0.2, 0.2, 0.2), 0.1, radius=0.05, environment=1)                 # 27 particles
    w.add_cloth_grid((4, 3), (0.3, 0.2), position=(1.0, 0.5, 0.0), radius=0.01, layer=2, mask=6)
    w.add_strand([(0.0, 1.0, 0.1 * k) for k in range(5)], radius=0.01, environment=2)
    w.add_strand([(0.5, 1.0, 0.1 * k) for k in range(3)], radius=0.01)
    w.add_fluid_grid((0.2, 0.1, 0.2), 0.05, position=(2.0, 0.5, 0.0), radius=0.03, environment=3)
    return w


def test_owner_ranges_and_particle_arrays():
    w = world()
    soa = w.soa()
    m = w.layout_mapping()
    n = soa.particle_count
    assert m["particle_count"] == n
    assert (m["soft_body_count"], m["cloth_count"], m["strand_count"], m["fluid_count"]) == (1, 1, 2, 1)
    sb, cl, st, fl = m["soft_bodies"], m["cloths"], m["strands"], m["fluids"]
    assert sb["particle_offsets"].tolist() == [0] and sb["particle_counts"].tolist() == [27]
    assert cl["particle_offsets"].tolist() == [27] and cl["particle_counts"].tolist() == [12]
    assert st["particle_offsets"].tolist() == [39, 44] and st["particle_counts"].tolist() == [5, 3]
    assert fl["particle_offsets"].tolist() == [47] and fl["particle_counts"][0] == n - 47
    assert sb["environment_indices"].tolist() == [1] and st["environment_indices"].tolist() == [2, 0]
    assert fl["environment_indices"].tolist() == [3]
    assert st["ids"].tolist() == [0, 1]
    types = m["owner_types"]
    assert (types[:27] == OWNER_SOFT).all() and (types[27:39] == OWNER_CLOTH).all()
    assert (types[39:47] == OWNER_STRAND).all() and (types[47:] == OWNER_FLUID).all()
    assert m["strand_ids"][39:44].tolist() == [0] * 5 and m["strand_ids"][44:47].tolist() == [1] * 3
    assert m["strand_orders"][39:47].tolist() == [0, 1, 2, 3, 4, 0, 1, 2]
    assert (m["strand_ids"][:39] == 0xFFFFFFFF).all() and (m["strand_orders"][47:] == 0xFFFFFFFF).all()
    assert (m["owning_soft_body_indices"][:27] == 0).all() and (m["owning_soft_body_indices"][27:] == 0xFFFFFFFF).all()
    assert (m["strand_roles"] == 0).all()
    meta = np.ctypeslib.as_array(soa.metadata, (n * 4,)).reshape(n, 4)
    assert np.array_equal(m["environment_indices"], meta[:, 0]) and np.array_equal(m["phases"], meta[:, 1])
    assert np.array_equal(m["collision_layers"], meta[:, 2]) and np.array_equal(m["collision_masks"], meta[:, 3])
    assert (m["collision_layers"][27:39] == 2).all() and (m["collision_masks"][27:39] == 6).all()
    assert np.array_equal(m["adjacency_counts"], np.ctypeslib.as_array(soa.adjacency_counts, (n,)))


def test_layout_revision_changes_with_a_new_packing():
    w = world()
    r0 = w.layout_mapping()["layout_revision"]
    assert w.layout_mapping()["layout_revision"] == r0          # no authoring change: same packing
    w.add_strand([(3.0, 1.0, 0.1 * k) for k in range(4)], radius=0.01)
    m = w.layout_mapping()
    assert m["layout_revision"] != r0 and m["strand_count"] == 3
