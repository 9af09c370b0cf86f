"""Surface render passes: render-mesh binding on the host (world.cpp:180-395, 3255-3554), the
skinning / normal / bounds passes (physics/soft/render/ shaders) in the oracle, and the sm_100a
kernels against the oracle (bit-exact: the passes use only + - * / sqrt, min and max)."""
import numpy as np
import pytest

from cn_physics import CNError, Solver, World, scenes, solver_desc
import cn_oracle


def block_world(meshfree=False, cloth=True):
    w = World()
    size, spacing = (0.5, 0.25, 0.375), 0.125
    w.add_soft_body_grid(size, spacing, position=(0.0, 0.4, 0.0), radius=0.05, edge_compliance=1e-5,
                         volume_compliance=1e-6)
    pos, tri, nrm = scenes.grid_surface_mesh(size, spacing)
    first = w.add_surface_mesh("soft_body", 0, pos, tri, nrm)
    if cloth:
        c = w.add_cloth_grid((6, 5), (0.5, 0.4), position=(0.0, 0.9, 0.0), radius=0.02,
                             structural_compliance=1e-6, static_particles=[0, 5])
        cx, cz = np.meshgrid((np.arange(6) / 5.0 - 0.5) * 0.5, (np.arange(5) / 4.0 - 0.5) * 0.4, indexing="xy")
        cloth_pos = np.stack([cx.ravel(), np.zeros(30), cz.ravel()], 1).astype(np.float32)
        ctri = []
        for j in range(4):
            for i in range(5):
                a, b, cc, d = j * 6 + i, j * 6 + i + 1, (j + 1) * 6 + i + 1, (j + 1) * 6 + i
                ctri += [(a, b, cc), (a, cc, d)]
        w.add_surface_mesh("cloth", c, cloth_pos, np.array(ctri, np.uint32))
    if meshfree:
        rng = np.random.default_rng(3)
        pts = rng.uniform(-0.15, 0.15, size=(60, 3)).astype(np.float32)
        mf = w.add_soft_body_meshfree(pts, 6, position=(0.6, 0.5, 0.0), radius=0.03, edge_compliance=1e-5)
        verts = rng.uniform(-0.12, 0.12, size=(20, 3)).astype(np.float32)
        vt = np.array([(k, k + 1, k + 2) for k in range(0, 18, 3)], np.uint32)
        w.add_surface_mesh("soft_body", mf, verts, vt)
    scenes.ground(w)
    return w, first, (pos, tri, nrm)


def surface_arrays(soa):
    sr = soa.surface_render.contents
    V, T, S = sr.vertex_count, sr.triangle_count, sr.surface_count
    b = np.ctypeslib.as_array(C_cast(sr.vertex_bindings, 8 * V), (V * 8,)).view(np.uint32).reshape(V, 8)
    ranges = np.ctypeslib.as_array(C_cast(sr.vertex_triangle_ranges, 4 * V), (V * 4,)).view(np.uint32).reshape(V, 4)
    idx = np.ctypeslib.as_array(sr.vertex_triangle_indices, (sr.vertex_triangle_index_count,))
    tri = np.ctypeslib.as_array(sr.triangle_particle_indices, (T * 4,)).reshape(T, 4)
    surf = np.ctypeslib.as_array(sr.surface_particle_ranges, (S * 2,)).reshape(S, 2)
    return b, ranges, idx, tri, surf


def C_cast(ptr, n):
    import ctypes as C
    return C.cast(ptr, C.POINTER(C.c_uint32))


def test_exact_bindings_triangles_and_incidence():
    w, first, (pos, tri, _) = block_world()
    soa = w.soa()
    b, ranges, idx, tris, surf = surface_arrays(soa)
    assert first == 0
    x = w.positions()[:, :3]
    # exact binding: the vertex sits on its particle (object frame + the body's translation)
    p = b[: pos.shape[0], 0]
    assert (b[: pos.shape[0], 1:4] == p[:, None]).all()
    w0 = b[: pos.shape[0], 4:].view(np.float32)
    assert (w0[:, 0] == 1.0).all() and (w0[:, 1:] == 0.0).all()
    assert np.abs(x[p] - (pos + np.float32([0.0, 0.4, 0.0]))).max() < 1e-6
    # triangles use the dominant particles of their vertices; incident lists in triangle order
    assert (tris[: tri.shape[0], :3] == p[tri]).all()
    for v in range(b.shape[0]):
        lst = idx[ranges[v, 0]: ranges[v, 0] + ranges[v, 1]]
        assert (np.diff(lst) > 0).all()
    counts = np.bincount(idx, minlength=tris.shape[0])
    assert (counts == 3).all()
    # one surface per soft body and cloth, packed [soft bodies][cloths]
    assert surf.tolist() == [[0, 5 * 3 * 4], [60, 30]]


def test_nearest_particle_bindings_for_meshfree():
    w, _, _ = block_world(meshfree=True)
    soa = w.soa()
    b, *_ = surface_arrays(soa)
    x = w.positions()[:, :3]
    mf_off, mf_n = 60, 60   # soft bodies pack before cloths
    verts = b[-20:]
    idx4 = verts[:, :4]
    wts = verts[:, 4:].view(np.float32)
    assert ((idx4 >= mf_off) & (idx4 < mf_off + mf_n)).all()
    assert np.allclose(wts.sum(1), 1.0, atol=1e-6)
    # weights fall with distance, the 4 nearest rest particles (restated with numpy)
    rng = np.random.default_rng(3)
    pts = rng.uniform(-0.15, 0.15, size=(60, 3)).astype(np.float32)
    vq = rng.uniform(-0.12, 0.12, size=(20, 3)).astype(np.float32)
    for k in range(20):
        d = ((pts - vq[k]) ** 2).sum(1)
        want = np.argsort(d, kind="stable")[:4] + mf_off
        assert sorted(want.tolist()) == sorted(idx4[k].tolist())
        assert (np.diff(wts[k]) <= 0).all()


def test_binding_errors():
    w = World()
    w.add_soft_body_grid((0.5, 0.5, 0.5), 0.25)
    with pytest.raises(CNError):
        w.add_surface_mesh("soft_body", 0, np.array([[0.1, 0.1, 0.1]], np.float32), np.zeros((0, 3), np.uint32))
    with pytest.raises(CNError):
        w.add_surface_mesh("soft_body", 3, np.zeros((1, 3), np.float32), np.zeros((0, 3), np.uint32))
    c = w.add_cloth_grid((3, 3), (1.0, 1.0))
    cp = np.array([[-0.5, 0, -0.5], [0.0, 0, -0.5], [0.0, 0, -0.5]], np.float32)
    with pytest.raises(CNError):   # two vertices on one particle collapse the triangle
        w.add_surface_mesh("cloth", c, cp, np.array([[0, 1, 2]], np.uint32))


def test_oracle_surface_passes():
    w, _, (pos, tri, _) = block_world()
    desc = solver_desc(substeps=2)
    soa = w.soa()
    ora = cn_oracle.Oracle(desc, soa)
    for _ in range(3):
        ora.step(1.0 / 60.0)
    rp, rn, box, tn = ora.read_surface_render()
    x, _, _ = ora.read_particles()
    b, ranges, idx, tris, surf = surface_arrays(soa)
    # exact bindings skin to the particle positions bit for bit
    assert np.array_equal(rp[:, :3], x[b[:, 0], :3]) and (rp[:, 3] == 1.0).all()
    assert np.allclose(np.linalg.norm(rn[:, :3], axis=1), 1.0, atol=1e-6)
    for k, (o, n) in enumerate(surf):
        assert np.array_equal(box[k, :3], x[o:o + n, :3].min(0)) and np.array_equal(box[k, 4:7], x[o:o + n, :3].max(0))
    # face normals point out of the block
    p0, p1, p2 = (x[tris[: tri.shape[0], k], :3] for k in range(3))
    cen = x[:60, :3].mean(0)
    assert ((tn[: tri.shape[0], :3] * ((p0 + p1 + p2) / 3 - cen)).sum(1) > 0).all()


def restated_surface(x, b, ranges, idx, tris, fallback, surf):
    """numpy float32 restatement of the passes in the shaders' operation order."""
    f = np.float32
    wts = b[:, 4:].view(np.float32)
    acc = np.zeros((b.shape[0], 3), f)
    for k in range(4):
        acc = acc + wts[:, k:k + 1] * x[b[:, k], :3]
    p0, p1, p2 = (x[tris[:, k], :3] for k in range(3))
    e1, e2 = p2 - p0, p1 - p0
    tn = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1], e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                   e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], 1)
    nrm = np.zeros((b.shape[0], 3), f)
    for v in range(b.shape[0]):
        a = np.zeros(3, f)
        for t in idx[ranges[v, 0]: ranges[v, 0] + ranges[v, 1]]:
            a = a + tn[t]
        l2 = f(a[0] * a[0] + a[1] * a[1]) + f(a[2] * a[2])
        nrm[v] = fallback[v, :3] if l2 <= f(1e-12) else a * (f(1.0) / np.sqrt(l2))
    box = np.zeros((surf.shape[0], 8), f)
    for k, (o, n) in enumerate(surf):
        if n:
            box[k, :3], box[k, 4:7] = x[o:o + n, :3].min(0), x[o:o + n, :3].max(0)
    return acc, nrm, box


@pytest.mark.gpu
def test_surface_passes_on_cloth_and_block_match_restatement():
    """With cloth (its dihedral solve holds the 1e-5 tolerance, not bits) the passes are checked
    against a restatement on the GPU's own positions."""
    w, _, _ = block_world(meshfree=False, cloth=True)
    soa = w.soa()
    gpu = Solver(solver_desc(substeps=4))
    gpu.sync_world(soa)
    for _ in range(8):
        gpu.step(1.0 / 60.0)
    x, _, _ = gpu.read_particles()
    b, ranges, idx, tris, surf = surface_arrays(soa)
    fb = np.ctypeslib.as_array(soa.surface_render.contents.fallback_normals, (b.shape[0] * 4,)).reshape(-1, 4)
    rp, rn, rb = restated_surface(x, b, ranges, idx, tris, fb, surf)
    gp, gn, gb = gpu.read_surface_render()
    assert np.array_equal(gp[:, :3], rp) and (gp[:, 3] == 1.0).all()
    assert np.array_equal(gb, rb)
    assert np.abs(gn[:, :3] - rn).max() <= 1e-6   # sum of three squares may associate differently


@pytest.mark.gpu
@pytest.mark.parametrize("meshfree", [False, True])
def test_surface_passes_bit_exact_with_oracle(meshfree):
    w, _, _ = block_world(meshfree, cloth=False)
    desc = solver_desc(substeps=4)
    soa = w.soa()
    gpu = Solver(desc)
    gpu.sync_world(soa)
    ora = cn_oracle.Oracle(desc, soa)
    for _ in range(10):
        gpu.step(1.0 / 60.0)
        ora.step(1.0 / 60.0)
    xg, _, _ = gpu.read_particles()
    xo, _, _ = ora.read_particles()
    assert np.array_equal(xg, xo)
    gp, gn, gb = gpu.read_surface_render()
    op, on, ob, _ = ora.read_surface_render()
    assert np.array_equal(gp, op) and np.array_equal(gn, on) and np.array_equal(gb, ob)
    v = gpu.surface_render_view()
    surf = surface_arrays(soa)[4]
    assert v["vertex_count"] == gp.shape[0] and v["surface_count"] == gb.shape[0]
    assert v["chunk_count"] == sum((int(n) + 63) // 64 for _, n in surf)


@pytest.mark.gpu
def test_surface_render_dlpack_and_update():
    import torch
    w, _, _ = block_world()
    soa = w.soa()
    gpu = Solver(solver_desc(substeps=2))
    gpu.sync_world(soa)
    gpu.step(1.0 / 60.0)
    t = gpu.export_dlpack("render_positions")
    pos, _, box = gpu.read_surface_render()
    assert torch.equal(t.cpu(), torch.from_numpy(pos))
    tb = gpu.export_dlpack("surface_world_aabbs")
    assert tuple(tb.shape) == box.shape and torch.equal(tb.cpu(), torch.from_numpy(box))
    # same counts, new fallback normals: uploaded in place
    b, ranges, idx, tris, surf = surface_arrays(soa)
    fn = np.ctypeslib.as_array(soa.surface_render.contents.fallback_normals, (b.shape[0] * 4,))
    fn[:] = 0.0
    gpu.update_world(soa, "surface_render")
    gpu.step(1.0 / 60.0)
    assert np.isfinite(gpu.read_surface_render()[1]).all()
