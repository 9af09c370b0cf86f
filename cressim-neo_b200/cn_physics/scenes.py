"""Seeded synthetic scenes for the reference's benchmark configurations.

No public dataset is involved: every scene is generated from its sizes and a seed, with the
shapes and value ranges of the configurations it stands for.

* ``xpbd_cube``   -- plain XPBD soft body: 16x16x16-vertex lattice split 5 tets per cell
                     (16,875 tets), edge compliance 1e-5, volume compliance 1e-6, bottom face
                     pinned, ground box with its top face at y = 0, jitter +-1e-3 of the edge length.
* ``dam_break``   -- plain PBF dam break: 128x64x128 fluid lattice (1,048,576 particles) at spacing
                     0.05 (h = 0.1, radius 0.03) in a 12.8 x 6.4 x 25.6 box of static walls,
                     viscosity 0.01, vorticity off, jitter +-1e-4.
* ``mixed_surgical`` -- tissue lattice + cloth + strands + fluid block + a kinematic capsule tool,
                        render meshes on the tissue and the cloth.
"""
from __future__ import annotations

import math

import numpy as np

from . import World, solver_desc


def _jitter(world: World, amplitude: float, seed: int) -> None:
    x = world.positions()
    rng = np.random.default_rng(seed)
    movable = x[:, 3] > 0.0
    j = rng.uniform(-amplitude, amplitude, size=(x.shape[0], 3)).astype(np.float32)
    x[movable, :3] += j[movable]


def grid_surface_mesh(size, spacing):
    """Boundary render mesh of a regular-grid soft body in its object frame: the lattice points of
    buildRegularGridSource (soft_body_authoring.cpp:81-176) on the six faces, two triangles per
    face cell wound so that cross(p2 - p0, p1 - p0) (the reference's face normal) points outward.
    Returns (positions (V, 3), triangles (F, 3), normals (V, 3))."""
    f = np.float32
    ext = [max(f(e), f(1e-4)) for e in size]
    sp = max(f(spacing), f(1e-4))
    res = [max(2, int(math.ceil(f(e) / sp)) + 1) for e in ext]
    rx, ry, rz = res
    coords = [((np.arange(n, dtype=f) / f(n - 1)) - f(0.5)) * e for n, e in zip(res, ext)]
    index = {}
    pos, nrm = [], []

    def vid(i, j, k, n):
        key = (i, j, k)
        if key not in index:
            index[key] = len(pos)
            pos.append((coords[0][i], coords[1][j], coords[2][k]))
            nrm.append(n)
        return index[key]

    tris = []
    # each face: (fixed axis, fixed value index, outward sign)
    for axis in range(3):
        for side, sign in ((0, -1.0), (res[axis] - 1, 1.0)):
            a, b = [d for d in range(3) if d != axis]
            n = [0.0, 0.0, 0.0]
            n[axis] = sign
            for u in range(res[a] - 1):
                for v in range(res[b] - 1):
                    corner = []
                    for du, dv in ((0, 0), (1, 0), (1, 1), (0, 1)):
                        ijk = [0, 0, 0]
                        ijk[axis], ijk[a], ijk[b] = side, u + du, v + dv
                        corner.append(vid(*ijk, tuple(n)))
                    q0, q1, q2, q3 = corner
                    # cross(p2 - p0, p1 - p0) along +axis for (q0, q3, q2) when a < b
                    outward_ccw = (sign > 0) == ((axis == 1))
                    if outward_ccw:
                        tris += [(q0, q1, q2), (q0, q2, q3)]
                    else:
                        tris += [(q0, q2, q1), (q0, q3, q2)]
    return np.array(pos, np.float32), np.array(tris, np.uint32), np.array(nrm, np.float32)


def ground(world: World, top_y: float = 0.0, half=(50.0, 0.5, 50.0), friction=0.5) -> int:
    body = world.add_rigid_body("static", position=(0.0, top_y - half[1], 0.0))
    world.add_collider(body, "box", half, friction=friction)
    return body


def xpbd_cube(n: int = 16, spacing: float = 1.0 / 16.0, seed: int = 0, radius: float | None = None,
              pin_bottom: bool = True, lift: float = 0.0):
    """Returns (world, desc, frame_dt).  n vertices per axis; cube bottom face sits on the ground."""
    w = World()
    size = (n - 1) * spacing
    r = spacing * 0.5 if radius is None else radius
    res = n
    static = []
    if pin_bottom:
        for x in range(res):
            for z in range(res):
                static.append(x * res * res + 0 * res + z)
    w.add_soft_body_grid((size, size, size), spacing, position=(0.0, size * 0.5 + r + lift, 0.0),
                         radius=r, edge_compliance=1.0e-5, volume_compliance=1.0e-6,
                         static_particles=static, friction=0.3)
    ground(w)
    w.soa()
    _jitter(w, 1.0e-3 * spacing, seed)
    desc = solver_desc(substeps=10, default_iterations=20, enable_blocking_readback=0)
    return w, desc, 1.0 / 60.0


def dam_break(nx: int = 128, ny: int = 64, nz: int = 128, spacing: float = 0.05, seed: int = 0,
              box=(12.8, 6.4, 25.6), vorticity: float = 0.0):
    """Returns (world, desc, frame_dt)."""
    w = World()
    r = 0.6 * spacing  # h = max((2/0.6) r, 2r) = 2 * spacing
    size = (nx * spacing, ny * spacing, nz * spacing)
    offset = r - 0.5 * spacing
    center = (size[0] * 0.5 + offset, size[1] * 0.5 + offset, size[2] * 0.5 + offset)
    w.add_fluid_grid(size, spacing, position=center, radius=r, viscosity=0.01, vorticity=vorticity)
    body = w.add_rigid_body("static")
    bx, by, bz = box
    t = 0.5
    w.add_collider(body, "box", (bx * 0.5 + 2 * t, t, bz * 0.5 + 2 * t), (bx * 0.5, -t, bz * 0.5))
    w.add_collider(body, "box", (t, by * 0.5 + 2 * t, bz * 0.5 + 2 * t), (-t, by * 0.5, bz * 0.5))
    w.add_collider(body, "box", (t, by * 0.5 + 2 * t, bz * 0.5 + 2 * t), (bx + t, by * 0.5, bz * 0.5))
    w.add_collider(body, "box", (bx * 0.5 + 2 * t, by * 0.5 + 2 * t, t), (bx * 0.5, by * 0.5, -t))
    w.add_collider(body, "box", (bx * 0.5 + 2 * t, by * 0.5 + 2 * t, t), (bx * 0.5, by * 0.5, bz + t))
    w.soa()
    _jitter(w, 1.0e-4, seed)
    desc = solver_desc(substeps=2, fluid_iterations=4, enable_blocking_readback=0)
    return w, desc, 1.0 / 120.0


def tool_path(t: float, seed: int = 0, center=(0.0, 0.6, 0.0), amplitude=0.3):
    """Seeded smooth random path: a sum of three sines per axis."""
    rng = np.random.default_rng(seed)
    freq = rng.uniform(0.3, 1.5, size=(3, 3))
    phase = rng.uniform(0.0, 2.0 * math.pi, size=(3, 3))
    amp = rng.uniform(0.3, 1.0, size=(3, 3))
    amp = amp / amp.sum(axis=1, keepdims=True) * amplitude
    p = [center[a] + float(np.sum(amp[a] * np.sin(freq[a] * t + phase[a]))) for a in range(3)]
    return tuple(p)


def cloth_grid_mesh(resolution, size):
    """Render mesh of a cloth grid in its own frame: one vertex per particle (the identity
    mapping of world.cpp:3300-3313) and the grid's triangles (v00, v10, v11), (v00, v11, v01)."""
    nx, ny = max(resolution[0], 2), max(resolution[1], 2)
    f = np.float32
    gx = (np.arange(nx, dtype=f) / f(nx - 1) - f(0.5)) * f(size[0])
    gz = (np.arange(ny, dtype=f) / f(ny - 1) - f(0.5)) * f(size[1])
    xx, zz = np.meshgrid(gx, gz, indexing="xy")
    pos = np.stack([xx.ravel(), np.zeros(nx * ny, f), zz.ravel()], 1)
    j, i = np.meshgrid(np.arange(ny - 1), np.arange(nx - 1), indexing="ij")
    v00 = (j * nx + i).ravel()
    v10, v01, v11 = v00 + 1, v00 + nx, v00 + nx + 1
    tri = np.concatenate([np.stack([v00, v10, v11], 1), np.stack([v00, v11, v01], 1)]).astype(np.uint32)
    return pos, tri


def mixed_surgical(tissue=(60, 30, 60), cloth=(256, 256), strands=(64, 129), fluid=(64, 64, 64),
                   seed: int = 0, surfaces: bool = True):
    """Tissue lattice + cloth sheet + strands + fluid block + kinematic capsule (r = 0.01), with
    render meshes on the tissue (its boundary faces) and the cloth when `surfaces`.
    Returns (world, desc, frame_dt, tool_body)."""
    w = World()
    sp = 0.02
    tx, ty, tz = tissue
    tsize = ((tx - 1) * sp, (ty - 1) * sp, (tz - 1) * sp)
    w.add_soft_body_grid(tsize, sp, position=(0.0, tsize[1] * 0.5 + 0.01, 0.0), radius=0.01,
                         edge_compliance=1.0e-5, volume_compliance=1.0e-6, friction=0.3)
    cres = cloth
    csize = (tsize[0] * 1.2, tsize[2] * 1.2)
    w.add_cloth_grid(cres, csize, position=(0.0, tsize[1] + 0.05, 0.0), radius=0.004,
                     structural_compliance=1.0e-6, bend_compliance=1.0e-3, friction=0.3)
    ns, npts = strands
    for k in range(ns):
        x0 = -tsize[0] * 0.5 + (k + 0.5) * tsize[0] / ns
        pts = [(x0, tsize[1] + 0.15, -tsize[2] * 0.5 + j * tsize[2] / (npts - 1)) for j in range(npts)]
        w.add_strand(pts, radius=0.003, stretch_shear_compliance=1.0e-6, bend_compliance=1.0e-4,
                     twist_compliance=1.0e-4, static_particles=[0])
    fx, fy, fz = fluid
    fsp = 0.01
    w.add_fluid_grid((fx * fsp, fy * fsp, fz * fsp), fsp,
                     position=(tsize[0] * 0.5 + 0.1 + fx * fsp * 0.5, fy * fsp * 0.5 + 0.01, 0.0),
                     radius=0.6 * fsp)
    ground(w)
    tool = w.add_rigid_body("kinematic", position=tool_path(0.0, seed))
    w.add_collider(tool, "capsule", (0.01, 0.1), friction=0.2)
    if surfaces:
        pos, tri, nrm = grid_surface_mesh(tsize, sp)
        w.add_surface_mesh("soft_body", 0, pos, tri, nrm)
        cpos, ctri = cloth_grid_mesh(cres, csize)
        w.add_surface_mesh("cloth", 0, cpos, ctri)
    w.soa()
    _jitter(w, 1.0e-4, seed)
    desc = solver_desc(substeps=8, enable_blocking_readback=0)
    return w, desc, 1.0 / 60.0, tool


def rigid_pile(layers: int = 4, per_side: int = 32, seed: int = 0, proxy_tools: int = 4):
    """Dynamic bodies dropped onto the ground in `layers` layers of per_side^2 (spheres, capsules and
    boxes in turn, seeded jitter), plus `proxy_tools` dynamic bodies made of 27 proxy particles each:
    the rigid broadphase (LBVH), the box-box manifold, depenetration and the body-pair velocity
    solve, and proxy contacts.  Returns (world, desc, frame_dt, bodies)."""
    rng = np.random.default_rng(seed)
    w = World()
    ground(w)
    bodies = []
    pitch = 0.12
    half = (per_side - 1) * pitch * 0.5
    k = 0
    for ly in range(layers):
        for ix in range(per_side):
            for iz in range(per_side):
                p = (ix * pitch - half + float(rng.uniform(-0.01, 0.01)), 0.06 + ly * pitch,
                     iz * pitch - half + float(rng.uniform(-0.01, 0.01)))
                b = w.add_rigid_body("dynamic", position=p, mass=0.2, inverse_inertia=(400.0,) * 3)
                if k % 3 == 0:
                    w.add_collider(b, "sphere", (0.04,), friction=0.5)
                elif k % 3 == 1:
                    w.add_collider(b, "capsule", (0.03, 0.03), friction=0.5)
                else:
                    w.add_collider(b, "box", (0.04, 0.04, 0.04), friction=0.5)
                bodies.append(b)
                k += 1
    g = (np.arange(3) - 1.0) * 0.04
    lattice = np.array([(x, y, z) for x in g for y in g for z in g], np.float32)
    for t in range(proxy_tools):
        p = (-half + (t + 0.5) * 2 * half / max(proxy_tools, 1), 0.3 + layers * pitch, 0.0)
        b = w.add_rigid_body("dynamic", position=p, mass=0.5, inverse_inertia=(800.0,) * 3)
        w.set_rigid_proxy_particles(b, lattice, 0.02, friction=0.5)
        bodies.append(b)
    w.soa()
    # the proxies sit in the pile against more bodies than the reference's 8 candidate pairs per
    # particle hold (~800 of 864 in the oracle's pile): 16 per particle
    desc = solver_desc(substeps=4, default_iterations=10, enable_blocking_readback=0,
                       particle_rigid_pairs_per_particle=16)
    return w, desc, 1.0 / 60.0, bodies
