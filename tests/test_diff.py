"""Differentiable XPBD rollout: forward bit-identical to the solver, adjoint against FP64
central finite differences (eps = 1e-6) on a ~2K-tet block, checkpoint-interval independence and
the torch.autograd.Function."""
import numpy as np
import pytest

from cn_physics import Solver, World, solver_desc
from cn_physics import diff
from conftest import has_gpu

DIMS = (9, 8, 8)                 # vertices: 8 * 7 * 7 cells * 5 = 1960 tets


# XPBD compliance is relative to the constraint's gradient: for 10 cm tets |grad V|^2 ~ 3e-6, and at
# dt = 1/480 s a compliance of 1e-11 gives alpha / dt^2 ~ 2e-6, so the volume constraints carry
# the block's stiffness (soft edges, compliance 1e-4) and the per-tet compliances are identifiable.
def block(dims=DIMS, spacing=0.1, seed=0, base=1e-11):
    rx, ry, rz = dims
    w = World()
    size = ((rx - 1.25) * spacing, (ry - 1.25) * spacing, (rz - 1.25) * spacing)
    pinned = [x * ry * rz + z for x in range(rx) for z in range(rz)]
    w.add_soft_body_grid(size, spacing, position=(0.0, size[1] * 0.5, 0.0), radius=0.4 * spacing,
                         edge_compliance=1e-4, volume_compliance=base, static_particles=pinned)
    w.soa()
    rng = np.random.default_rng(seed)
    comp = w.array("tets").view(np.float32)[:, 5]
    comp[:] = (base * rng.lognormal(0.0, 0.5, comp.shape[0])).astype(np.float32)
    return w


def test_surface_indices():
    s = diff.lattice_surface((3, 3, 3))
    assert len(s) == 26 and 13 not in s


def test_block_counts():
    w = block()
    c = w.counts()
    assert c["particles"] == 9 * 8 * 8 and c["tets"] == 1960


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_rollout_needs_a_device():
    from cn_physics import CNError
    with pytest.raises(CNError):
        diff.Rollout(block())


def _inputs(w, torch, dtype, seed=1):
    x0 = torch.as_tensor(w.positions().copy(), device="cuda", dtype=dtype)
    comp = torch.as_tensor(w.array("tets").view(np.float32)[:, 5].copy(), device="cuda", dtype=dtype)
    rng = np.random.default_rng(seed)
    v = np.zeros((x0.shape[0], 4))
    v[:, :3] = rng.normal(0.0, 0.05, (x0.shape[0], 3))
    v0 = torch.as_tensor(v, device="cuda", dtype=dtype)
    v0[x0[:, 3] <= 0] = 0
    return comp, x0, v0


@pytest.mark.gpu
def test_float_forward_is_the_solver_bit_for_bit():
    import torch
    w = block()
    substeps, iters, frame = 8, 10, 1.0 / 60.0
    sdt = float(np.float32(frame) / np.float32(substeps))
    r = diff.Rollout(w, substeps=substeps, iterations=iters, substep_dt=sdt, checkpoint_interval=4)
    comp, x0, v0 = _inputs(w, torch, torch.float32)
    out = torch.empty_like(x0)
    vout = torch.empty_like(x0)
    r.forward(comp, x0, v0, out, vout)
    torch.cuda.synchronize()
    soa = w.soa()
    w.velocities()[:] = v0.cpu().numpy()
    sv = Solver(solver_desc(substeps=substeps, default_iterations=iters, enable_blocking_readback=0))
    sv.sync_world(soa)
    sv.step(frame)
    xs, vs, _ = sv.read_particles()
    assert np.array_equal(out.cpu().numpy()[:, :3], xs[:, :3])
    assert np.array_equal(vout.cpu().numpy()[:, :3], vs[:, :3])


def _loss_and_grads(r, comp, x0, v0, target, surf, torch):
    out = torch.empty_like(x0)
    r.forward(comp, x0, v0, out)
    d = out[surf, :3] - target[surf, :3]
    loss = (d * d).mean()
    g = torch.zeros_like(out)
    g[surf, :3] = 2.0 * d / d.numel()
    gc, gx, gv = torch.zeros_like(comp), torch.zeros_like(x0), torch.zeros_like(v0)
    r.backward(g, None, gc, gx, gv)
    torch.cuda.synchronize()
    return float(loss), gc, gv


def _loss(r, comp, x0, v0, target, surf, torch):
    out = torch.empty_like(x0)
    r.forward(comp, x0, v0, out)
    d = out[surf, :3] - target[surf, :3]
    return float((d * d).mean())


@pytest.mark.gpu
def test_adjoint_matches_fp64_central_differences():
    import torch
    w = block()
    surf = torch.as_tensor(diff.lattice_surface(DIMS), device="cuda")
    kw = dict(substeps=32, iterations=10, substep_dt=1.0 / 480.0, checkpoint_interval=8)
    r64 = diff.Rollout(w, precision=8, **kw)
    comp, x0, v0 = _inputs(w, torch, torch.float64)
    rng = np.random.default_rng(7)
    target_comp = comp * torch.as_tensor(rng.lognormal(0.0, 0.3, comp.shape[0]), device="cuda")
    target = torch.empty_like(x0)
    r64.forward(target_comp, x0, v0, target)
    loss, gc, gv = _loss_and_grads(r64, comp, x0, v0, target, surf, torch)
    assert loss > 1e-12
    eps = 1e-6
    # directional derivatives: compliance in log space (scaled by the compliance), and velocities
    for k in range(3):
        u = torch.as_tensor(rng.normal(0.0, 1.0, comp.shape[0]), device="cuda") * comp
        fd = (_loss(r64, comp + eps * u, x0, v0, target, surf, torch) -
              _loss(r64, comp - eps * u, x0, v0, target, surf, torch)) / (2 * eps)
        an = float((gc * u).sum())
        assert abs(an - fd) <= 1e-5 * abs(fd) + 1e-14, (k, an, fd)
        uv = torch.zeros_like(v0)
        uv[:, :3] = torch.as_tensor(rng.normal(0.0, 1.0, (v0.shape[0], 3)), device="cuda")
        uv[x0[:, 3] <= 0] = 0
        fdv = (_loss(r64, comp, x0, v0 + eps * uv, target, surf, torch) -
               _loss(r64, comp, x0, v0 - eps * uv, target, surf, torch)) / (2 * eps)
        anv = float((gv * uv).sum())
        assert abs(anv - fdv) <= 1e-5 * abs(fdv) + 1e-14, (k, anv, fdv)
    # the float adjoint agrees with the FP64 differences to float accuracy
    r32 = diff.Rollout(w, precision=4, **kw)
    _, gc32, gv32 = _loss_and_grads(r32, comp.float(), x0.float(), v0.float(), target.float(), surf, torch)
    rel = float((gc32.double() - gc).norm() / gc.norm())
    # the velocity gradient is small next to float rounding of the trajectory: compare directions
    cosv = float((gv32.double() * gv).sum() / (gv32.double().norm() * gv.norm()))
    assert rel < 2e-2 and cosv > 0.99, (rel, cosv)


@pytest.mark.gpu
def test_checkpoint_interval_does_not_change_gradients():
    import torch
    w = block((6, 5, 5))
    surf = torch.as_tensor(diff.lattice_surface((6, 5, 5)), device="cuda")
    comp, x0, v0 = _inputs(w, torch, torch.float32)
    target = x0.clone()
    target[:, 1] -= 0.01
    res = []
    for interval in (1, 3, 8, 16):
        r = diff.Rollout(w, substeps=16, iterations=5, substep_dt=1.0 / 480.0, checkpoint_interval=interval)
        res.append(_loss_and_grads(r, comp, x0, v0, target, surf, torch))
        r.close()
    for loss, gc, gv in res[1:]:
        assert loss == res[0][0] and torch.equal(gc, res[0][1]) and torch.equal(gv, res[0][2])


@pytest.mark.gpu
def test_autograd_function_identifies_compliance():
    import torch
    w = block((7, 6, 6))
    surf = torch.as_tensor(diff.lattice_surface((7, 6, 6)), device="cuda")
    r = diff.Rollout(w, substeps=16, iterations=10, substep_dt=1.0 / 480.0, checkpoint_interval=8)
    comp, x0, v0 = _inputs(w, torch, torch.float32)
    rng = np.random.default_rng(3)
    true = comp * torch.as_tensor(rng.lognormal(0.0, 0.3, comp.shape[0]), device="cuda", dtype=torch.float32)
    with torch.no_grad():
        target = diff.XPBDRollout.apply(true, v0, x0, r)
    logc = torch.log(comp).clone().requires_grad_(True)
    opt = torch.optim.Adam([logc], lr=0.1)
    losses = []
    for _ in range(40):
        opt.zero_grad()
        x = diff.XPBDRollout.apply(torch.exp(logc), v0, x0, r)
        loss = ((x[surf, :3] - target[surf, :3]) ** 2).mean()
        loss.backward()
        opt.step()
        losses.append(float(loss.detach()))
    assert losses[0] > 1e-12 and losses[-1] < 0.75 * losses[0], losses
