"""Batched and served forms: scenes in one pool, stepped together, equal scenes stepped alone.

The per-element arithmetic of a batch tick is that of a solver of its own (the scene's indices
are only rebased), so every comparison below is bit for bit.
"""
import numpy as np
import pytest

from cn_physics import Batch, Server, Solver, batch_desc, serving
from cn_physics._abi import XPBD_COLOUR_GAUSS_SEIDEL, XPBD_COLOUR_JACOBI, XPBD_GATHER
from conftest import has_gpu

DT = 1.0 / 60.0


def small_pool(n=4, seed=3):
    return [serving.tissue_scene(dims, seed=seed + k) for k, dims in
            enumerate([(6, 4, 6), (9, 3, 5), (4, 4, 4), (7, 5, 8), (5, 6, 3), (8, 4, 6)][:n])]


def targets_for(scene, frames, seed):
    rng = np.random.default_rng(seed)
    pose = scene.tool_pose.copy()
    out = []
    for _ in range(frames):
        pose = pose + rng.normal(0.0, 0.002, 3).astype(np.float32)
        pose[1] = max(pose[1] - 0.002, 0.0)   # press down into the tissue
        out.append(np.concatenate([pose, [0.0, 0.0, 0.7071068, 0.7071068]]).astype(np.float32))
    return np.stack(out)


def solver_desc_with(schedule):
    d = serving.serving_solver_desc()
    d.soft.xpbd_schedule = schedule
    return d


def own_solver_run(scene, targets, desc=None):
    sv = Solver(desc if desc is not None else serving.serving_solver_desc())
    sv.sync_world(scene.world.soa())
    for tg in targets:
        sv.set_kinematic_target(scene.tool, tg[:3], tg[3:])
        sv.step(DT)
    x, v, _ = sv.read_particles()
    sv.close()
    return x, v


# Scenes 0 and 2 stepped every tick; 1 and 3 only on some ticks (they catch up afterwards).
MIXED_TICKS = [[0, 1, 2, 3], [0, 2], [0, 2, 3], [0, 1, 2], [0, 2], [0, 1, 2, 3], [1, 3], [1, 3], [1, 3], [1]]


def run_mixed_ticks(b, pool, ids, tg, frames):
    done = [0] * len(pool)
    for tick in MIXED_TICKS:
        step = [k for k in tick if done[k] < frames]
        for k in step:
            t = tg[k][done[k]]
            b.set_kinematic_target(ids[k], pool[k].tool, t[:3], t[3:])
        b.step([ids[k] for k in step], DT)
        for k in step:
            done[k] += 1
    assert done == [frames] * len(pool)


def test_pool_generator_counts():
    pool = serving.tissue_pool(6, seed=1, tet_range=(2000, 8000))
    for sc in pool:
        cx, cy, cz = sc.cells
        assert sc.tets == 5 * cx * cy * cz and sc.particles == (cx + 1) * (cy + 1) * (cz + 1)
        assert 1000 <= sc.tets <= 12000
    req = serving.poisson_requests(pool, steps_per_second=20000.0, duration_s=0.5, seed=2)
    frames = sum(r.steps for r in req)
    assert 8000 < frames < 12000 and all(1 <= r.steps <= 8 for r in req)
    assert all(a.arrival <= b.arrival for a, b in zip(req, req[1:]))


def test_batch_desc_defaults():
    d = batch_desc()
    assert d.max_scenes == 1024 and d.tile_elements == 256 and d.blocks_per_sm == 8
    assert d.solver.default_iterations == 20 and d.solver.enable_blocking_readback == 0


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_batch_create_fails_without_device():
    from cn_physics import CNError
    with pytest.raises(CNError):
        Batch(batch_desc(serving.serving_solver_desc()))


@pytest.mark.gpu
@pytest.mark.parametrize("cluster_ctas", [0, 1, 2, 4, 8])
def test_batched_scene_equals_its_own_solver_and_is_independent_of_the_mix(cluster_ctas):
    """cluster_ctas 0: the per-phase iteration kernels; else the persistent fused iterations with
    one cluster of that many CTAs per scene (8 substeps per tick: the scene counter is reset
    between substeps)."""
    pool = small_pool(4)
    frames = 6
    tg = [targets_for(sc, frames, seed=10 + k) for k, sc in enumerate(pool)]
    ref = [own_solver_run(sc, tg[k]) for k, sc in enumerate(pool)]
    b = Batch(batch_desc(serving.serving_solver_desc(), memory_budget_bytes=1 << 30, particle_capacity=20000,
                         fused_cluster_ctas=cluster_ctas))
    assert b.stats()["fused_cluster_ctas"] == cluster_ctas
    ids = [b.add_scene(sc.world.soa()) for sc in pool]
    run_mixed_ticks(b, pool, ids, tg, frames)
    for k in range(len(pool)):
        x, v = b.read_particles(ids[k])
        assert np.array_equal(x, ref[k][0]) and np.array_equal(v, ref[k][1]), f"scene {k}"
    b.close()


@pytest.mark.gpu
def test_autotune_keeps_state_and_results():
    pool = small_pool(3)
    tg = [targets_for(sc, 3, seed=20 + k) for k, sc in enumerate(pool)]
    ref = [own_solver_run(sc, tg[k]) for k, sc in enumerate(pool)]
    b = Batch(batch_desc(serving.serving_solver_desc(), memory_budget_bytes=1 << 30, particle_capacity=10000))
    ids = [b.add_scene(sc.world.soa()) for sc in pool]
    tune = b.autotune(ids, DT)
    assert tune["candidates"] and tune["tick_ms"] > 0
    fused = [c for c in tune["candidates"] if c[3] > 0]
    assert len(tune["candidates"]) == 16 + len(fused) and {c[3] for c in fused} <= {1, 2, 4, 8} and fused
    assert b.stats()["fused_cluster_ctas"] == tune["cluster_ctas"]
    for f in range(3):
        for k in range(len(pool)):
            b.set_kinematic_target(ids[k], pool[k].tool, tg[k][f][:3], tg[k][f][3:])
        b.step(ids, DT)
    for k in range(len(pool)):
        x, v = b.read_particles(ids[k])
        assert np.array_equal(x, ref[k][0]) and np.array_equal(v, ref[k][1])
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", [XPBD_COLOUR_JACOBI, XPBD_COLOUR_GAUSS_SEIDEL])
def test_batched_scene_equals_its_own_solver_under_coloured_schedules(schedule):
    """A batch created with a coloured schedule: one kernel per colour over the stepped scenes,
    each scene's colour-k constraints and colour-Jacobi window its own solver's.  A scene removed
    and a new one admitted into the freed colour tables also match."""
    pool = small_pool(5)
    frames = 5
    desc = solver_desc_with(schedule)
    tg = [targets_for(sc, frames, seed=30 + k) for k, sc in enumerate(pool)]
    ref = [own_solver_run(sc, tg[k], desc) for k, sc in enumerate(pool)]
    b = Batch(batch_desc(desc, memory_budget_bytes=1 << 30, particle_capacity=30000))
    assert b.stats()["xpbd_schedule"] == schedule
    ids = [b.add_scene(sc.world.soa()) for sc in pool[:4]]
    run_mixed_ticks(b, pool[:4], ids, tg[:4], frames)
    for k in range(4):
        x, v = b.read_particles(ids[k])
        assert np.array_equal(x, ref[k][0]) and np.array_equal(v, ref[k][1]), f"scene {k}"
    b.remove_scene(ids[1])
    new = b.add_scene(pool[4].world.soa())
    for f in range(frames):
        b.set_kinematic_target(new, pool[4].tool, tg[4][f][:3], tg[4][f][3:])
        b.step([new, ids[0]], DT)
    x, v = b.read_particles(new)
    assert np.array_equal(x, ref[4][0]) and np.array_equal(v, ref[4][1])
    b.close()


@pytest.mark.gpu
def test_coloured_batch_switches_to_gather_and_autotune_picks_a_schedule():
    """A colour-Jacobi batch also runs the gather schedule (bit-identical to gather solvers); its
    autotuner times both and the chosen one still equals its solvers bit for bit; colour Jacobi
    and gather agree within 1e-5 (only the order of each particle's sum differs)."""
    pool = small_pool(3)
    frames = 3
    tg = [targets_for(sc, frames, seed=40 + k) for k, sc in enumerate(pool)]
    ref = {s: [own_solver_run(sc, tg[k], solver_desc_with(s)) for k, sc in enumerate(pool)]
           for s in (XPBD_GATHER, XPBD_COLOUR_JACOBI)}
    for k in range(len(pool)):
        np.testing.assert_allclose(ref[XPBD_COLOUR_JACOBI][k][0], ref[XPBD_GATHER][k][0], rtol=0, atol=1e-5)
    b = Batch(batch_desc(solver_desc_with(XPBD_COLOUR_JACOBI), memory_budget_bytes=1 << 30,
                         particle_capacity=10000))
    ids = [b.add_scene(sc.world.soa()) for sc in pool]
    tune = b.autotune(ids, DT)
    cands = tune["candidates"]
    cj = [c for c in cands if c[4] == XPBD_COLOUR_JACOBI]
    assert len(cj) == 4 and all(c[3] == 0 for c in cj), cands
    assert tune["xpbd_schedule"] in (XPBD_GATHER, XPBD_COLOUR_JACOBI)
    assert b.stats()["xpbd_schedule"] == tune["xpbd_schedule"]
    for mode in (XPBD_GATHER, XPBD_COLOUR_JACOBI):
        b.set_fused(0)
        b.set_xpbd_schedule(mode)
        ids2 = [b.add_scene(sc.world.soa()) for sc in pool]
        for f in range(frames):
            for k in range(len(pool)):
                b.set_kinematic_target(ids2[k], pool[k].tool, tg[k][f][:3], tg[k][f][3:])
            b.step(ids2, DT)
        for k in range(len(pool)):
            x, v = b.read_particles(ids2[k])
            assert np.array_equal(x, ref[mode][k][0]) and np.array_equal(v, ref[mode][k][1]), (mode, k)
            b.remove_scene(ids2[k])
    b.close()


@pytest.mark.gpu
def test_gather_batch_refuses_coloured_schedules():
    from cn_physics import CNError
    b = Batch(batch_desc(serving.serving_solver_desc(), memory_budget_bytes=1 << 28, particle_capacity=4000))
    with pytest.raises(CNError):
        b.set_xpbd_schedule(XPBD_COLOUR_JACOBI)
    b.set_xpbd_schedule(XPBD_GATHER)
    b.close()
    with pytest.raises(CNError):   # the fused iterations run the gather schedule
        Batch(batch_desc(solver_desc_with(XPBD_COLOUR_JACOBI), memory_budget_bytes=1 << 28,
                         particle_capacity=4000, fused_cluster_ctas=2))


@pytest.mark.gpu
def test_server_results_equal_alone_and_in_the_mix_with_evictions():
    pool = small_pool(6)
    # a budget that holds two or three of the six scenes: admissions must evict idle scenes
    # (the batch charges 120 + 4 x 72 B per particle, 60 B per edge, 116 B per tet, 272 B per
    # body and 216 B per collider)
    def scene_bytes(sc):
        c = sc.world.counts()
        return c["particles"] * (120 + 288) + c["edges"] * 60 + c["tets"] * 116 + 2 * 272 + 2 * 216
    largest = max(scene_bytes(sc) for sc in pool)
    b = Batch(batch_desc(serving.serving_solver_desc(), memory_budget_bytes=int(2.5 * largest),
                         particle_capacity=20000))
    srv = Server(b, DT)
    ids = [srv.register(sc.world.soa()) for sc in pool]
    req = serving.poisson_requests(pool, steps_per_second=600.0, duration_s=0.15, seed=5)
    per_scene = {k: [] for k in range(len(pool))}
    for r in req:
        per_scene[r.scene].append(r.targets)
    out = serving.serve(srv, pool, ids, req)
    st = out["stats"]
    assert out["requests"] == len(req) and st["pending"] == 0 and st["completed"] == len(req)
    assert st["evictions"] > 0, st
    for k, sc in enumerate(pool):
        if not per_scene[k]:
            continue
        tg = np.concatenate(per_scene[k])
        x_ref, v_ref = own_solver_run(sc, tg)
        x, v = srv.read_particles(ids[k])
        assert np.array_equal(x, x_ref) and np.array_equal(v, v_ref), f"scene {k}"
    srv.close()
    b.close()


@pytest.mark.gpu
def test_server_over_a_gauss_seidel_batch_with_evictions_equals_own_solvers():
    """The server's admission images carry the colourings when its batch runs a coloured schedule:
    scenes evicted and admitted again under a budget of about two scenes still equal solvers of
    their own under Gauss-Seidel."""
    pool = small_pool(6)
    desc = solver_desc_with(XPBD_COLOUR_GAUSS_SEIDEL)

    def scene_bytes(sc):   # the gather budget terms plus colour orders, sums and tables
        c = sc.world.counts()
        return (c["particles"] * (120 + 288 + 16) + c["edges"] * (60 + 16) + c["tets"] * (116 + 96)
                + 2 * 272 + 2 * 216 + 4 * 200)
    largest = max(scene_bytes(sc) for sc in pool)
    b = Batch(batch_desc(desc, memory_budget_bytes=int(2.5 * largest), particle_capacity=20000))
    srv = Server(b, DT)
    ids = [srv.register(sc.world.soa()) for sc in pool]
    # the request stream of the gather server test, which evicts under this budget
    req = serving.poisson_requests(pool, steps_per_second=600.0, duration_s=0.15, seed=5)
    per_scene = {k: [] for k in range(len(pool))}
    for r in req:
        per_scene[r.scene].append(r.targets)
    out = serving.serve(srv, pool, ids, req)
    st = out["stats"]
    assert out["requests"] == len(req) and st["pending"] == 0 and st["evictions"] > 0, st
    for k, sc in enumerate(pool):
        if not per_scene[k]:
            continue
        x_ref, v_ref = own_solver_run(sc, np.concatenate(per_scene[k]), desc)
        x, v = srv.read_particles(ids[k])
        assert np.array_equal(x, x_ref) and np.array_equal(v, v_ref), f"scene {k}"
    srv.close()
    b.close()


def serve_in_groups(srv, pool, ids, req, group, ticks_between):
    """Submits `group` requests, then ticks `ticks_between` times, until all are done: a fixed
    interleaving of submissions, admissions, evictions and ticks (no wall clock)."""
    nxt = 0
    while nxt < len(req) or srv.stats()["pending"]:
        for _ in range(group):
            if nxt < len(req):
                r = req[nxt]
                srv.submit(ids[r.scene], r.steps, tool_body=pool[r.scene].tool, targets=r.targets)
                nxt += 1
        for _ in range(ticks_between):
            srv.tick(0)
    srv.drain(0)


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", [XPBD_GATHER, XPBD_COLOUR_GAUSS_SEIDEL])
def test_server_interleavings_with_evictions_equal_own_solvers(schedule):
    """Fixed interleavings in which a request's last frame empties a scene's queue while its tick
    is being assembled, and a later scene of the same tick needs room: the scene already in the
    tick is not evicted (it used to be, and its batch id went to the admitted scene, which the tick
    then stepped twice)."""
    pool = small_pool(6)
    desc = solver_desc_with(schedule)
    req = serving.poisson_requests(pool, steps_per_second=600.0, duration_s=0.15, seed=5)
    per_scene = {k: [] for k in range(len(pool))}
    for r in req:
        per_scene[r.scene].append(r.targets)
    ref = {k: own_solver_run(pool[k], np.concatenate(t), desc) for k, t in per_scene.items() if t}
    coloured = schedule != XPBD_GATHER

    def scene_bytes(sc):   # the batch's budget charge, with the colour tables under a coloured schedule
        c = sc.world.counts()
        return (c["particles"] * (120 + 288 + 16 * coloured) + c["edges"] * (60 + 16 * coloured)
                + c["tets"] * (116 + 96 * coloured) + 2 * 272 + 2 * 216 + 4 * 200 * coloured)
    largest = max(scene_bytes(sc) for sc in pool)
    for group, ticks_between in ((1, 1), (2, 2), (100, 1)):
        b = Batch(batch_desc(desc, memory_budget_bytes=int(2.5 * largest), particle_capacity=20000))
        srv = Server(b, DT)
        ids = [srv.register(sc.world.soa()) for sc in pool]
        serve_in_groups(srv, pool, ids, req, group, ticks_between)
        assert srv.stats()["evictions"] > 0
        for k, (x_ref, v_ref) in ref.items():
            x, v = srv.read_particles(ids[k])
            assert np.array_equal(x, x_ref) and np.array_equal(v, v_ref), (group, ticks_between, k)
        srv.close()
        b.close()


@pytest.mark.gpu
def test_batch_step_rejects_a_scene_listed_twice():
    from cn_physics import CNError
    pool = small_pool(2)
    b = Batch(batch_desc(serving.serving_solver_desc(), memory_budget_bytes=1 << 28, particle_capacity=4000))
    ids = [b.add_scene(sc.world.soa()) for sc in pool]
    with pytest.raises(CNError):
        b.step([ids[0], ids[1], ids[0]], DT)
    b.step(ids, DT)
    b.close()


@pytest.mark.gpu
@pytest.mark.parametrize("schedule", [XPBD_GATHER, XPBD_COLOUR_JACOBI])
def test_random_admissions_removals_and_step_subsets_equal_own_solvers(schedule):
    """Seeded random sequence of adds (fragmenting the pool's ranges and colour tables), removals,
    targets and step subsets over eight small scenes; every resident instance equals a solver of
    its own that ran the same frames with the same targets."""
    rng = np.random.default_rng(7)
    desc = solver_desc_with(schedule)
    dims = [(3, 3, 3), (5, 2, 4), (4, 4, 2), (2, 3, 6), (6, 2, 2), (3, 5, 3), (4, 2, 5), (2, 2, 2)]
    pool = [serving.tissue_scene(d, seed=50 + k) for k, d in enumerate(dims)]
    # room for about four of the eight scenes (589 particles, 1,260 tets in all)
    b = Batch(batch_desc(desc, memory_budget_bytes=1 << 28, particle_capacity=330, edge_capacity=2400,
                         tet_capacity=700, max_scenes=8))
    full = 0
    live = {}   # scene index -> (batch id, targets stepped so far)
    for op in range(60):
        k = int(rng.integers(len(pool)))
        if k not in live:
            try:
                live[k] = (b.add_scene(pool[k].world.soa()), [])
            except Exception:   # the pool is full: drop a random resident scene instead
                full += 1
                victim = int(rng.choice(list(live)))
                b.remove_scene(live.pop(victim)[0])
            continue
        if rng.random() < 0.15:
            b.remove_scene(live.pop(k)[0])
            continue
        step = [j for j in live if rng.random() < 0.6] or [k]
        for j in step:
            pose = pool[j].tool_pose + rng.normal(0.0, 0.003, 3).astype(np.float32)
            tg = np.concatenate([pose, [0.0, 0.0, 0.7071068, 0.7071068]]).astype(np.float32)
            b.set_kinematic_target(live[j][0], pool[j].tool, tg[:3], tg[3:])
            live[j][1].append(tg)
        b.step([live[j][0] for j in step], DT)
    checked = 0
    for k, (bid, tgs) in live.items():
        x, v = b.read_particles(bid)
        if tgs:
            x_ref, v_ref = own_solver_run(pool[k], np.stack(tgs), desc)
        else:
            sv = Solver(desc)
            sv.sync_world(pool[k].world.soa())
            x_ref, v_ref, _ = sv.read_particles()
            sv.close()
        assert np.array_equal(x, x_ref) and np.array_equal(v, v_ref), (k, len(tgs))
        checked += 1
    assert checked >= 2 and full >= 3, (checked, full)
    b.close()
