"""Differentiable XPBD rollout (cn_diff_*) and its torch.autograd.Function.

    rollout = Rollout(world, substeps=32, iterations=20, substep_dt=1/480, checkpoint_interval=8)
    x = XPBDRollout.apply(tet_compliance, v0, x0, rollout) # (N, 4) positions after the rollout
    loss = ((x[surface, :3] - target[surface, :3]) ** 2).mean()
    loss.backward()                                        # d loss / d compliance, d loss / d v0

The forward runs the soft substep of the particle path in float (bit-identical to the solver) or
double; the backward is the library's hand-written adjoint, with positions and velocities
checkpointed every `checkpoint_interval` substeps and the rest recomputed.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import World, _abi, _check, load


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream_handle() -> C.c_void_p:
    import torch
    h = torch.cuda.current_stream().cuda_stream
    # torch's default stream has handle 0; the C ABI reads NULL as "the engine's own stream", so
    # the legacy default stream is named explicitly (cudaStreamLegacy == 0x1).
    return C.c_void_p(h if h else 1)


def lattice_surface(dims) -> np.ndarray:
    """Indices of the boundary vertices of a regular-grid soft body (flat = x*ry*rz + y*rz + z)."""
    rx, ry, rz = dims
    x, y, z = np.meshgrid(np.arange(rx), np.arange(ry), np.arange(rz), indexing="ij")
    b = (x == 0) | (x == rx - 1) | (y == 0) | (y == ry - 1) | (z == 0) | (z == rz - 1)
    return (x * ry * rz + y * rz + z)[b].astype(np.int64)


class Rollout:
    """One scene's differentiable rollout on the GPU."""

    def __init__(self, world: "World | _abi.WorldSoA", substeps: int = 32, iterations: int = 20,
                 substep_dt: float = 1.0 / 480.0, checkpoint_interval: int = 8, precision: int = 4,
                 gravity=(0.0, -9.81, 0.0), relaxation: float = 0.2, device: int = 0):
        self._lib = load()
        d = _abi.DiffDesc()
        self._lib.cn_diff_desc_defaults(C.byref(d))
        d.gravity = (C.c_float * 3)(*gravity)
        d.substeps, d.iterations = substeps, iterations
        d.substep_dt, d.relaxation = substep_dt, relaxation
        d.checkpoint_interval, d.precision = checkpoint_interval, precision
        self.desc = d
        h = C.c_void_p()
        _check(self._lib.cn_diff_create(C.byref(d), device, C.byref(h)))
        self._h = h
        soa = world.soa() if isinstance(world, World) else world
        _check(self._lib.cn_diff_set_scene(self._h, C.byref(soa)))
        self.n = soa.particle_count
        self.tets = soa.tet_count
        self.dtype = np.float64 if precision == 8 else np.float32

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cn_diff_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def memory_bytes(self) -> int:
        b = C.c_uint64()
        _check(self._lib.cn_diff_memory(self._h, C.byref(b)))
        return b.value

    def forward(self, compliance, x0, v0, x_out, v_out=None) -> None:
        """Device tensors: compliance (T,), x0 / v0 / x_out / v_out (N, 4), all of this rollout's dtype."""
        _check(self._lib.cn_diff_forward(self._h, _ptr(compliance), _ptr(x0), _ptr(v0), _ptr(x_out), _ptr(v_out),
                                         _stream_handle()))

    def backward(self, grad_x_out, grad_v_out, grad_compliance, grad_x0=None, grad_v0=None) -> None:
        _check(self._lib.cn_diff_backward(self._h, _ptr(grad_x_out), _ptr(grad_v_out), _ptr(grad_compliance),
                                          _ptr(grad_x0), _ptr(grad_v0), _stream_handle()))


def _autograd_function():
    import torch

    class XPBDRollout(torch.autograd.Function):
        """x_out = rollout(compliance, v0, x0): positions (N, 4; w = inverse mass) after the rollout.

        Gradients flow to the per-tet compliances, the initial velocities and the initial
        positions (the w column of x0 carries no gradient)."""

        @staticmethod
        def forward(ctx, compliance, v0, x0, rollout: Rollout):
            comp = compliance.detach().contiguous()
            v = v0.detach().contiguous()
            x = x0.detach().contiguous()
            out = torch.empty_like(x)
            rollout.forward(comp, x, v, out)
            ctx.rollout = rollout
            ctx.save_for_backward(comp, x, v)
            # the adjoint state the rollout holds belongs to its latest forward
            rollout._generation = getattr(rollout, "_generation", 0) + 1
            ctx.generation = rollout._generation
            return out

        @staticmethod
        def backward(ctx, grad_x):
            rollout = ctx.rollout
            comp, x, v = ctx.saved_tensors
            if getattr(rollout, "_generation", 0) != ctx.generation:
                rollout.forward(comp, x, v, torch.empty_like(x))  # another forward ran since
                rollout._generation += 1
                ctx.generation = rollout._generation
            gc = torch.zeros_like(comp)
            gv = torch.zeros_like(v)
            gx0 = torch.zeros_like(x)
            rollout.backward(grad_x.contiguous(), None, gc, gx0, gv)
            gx0[:, 3] = 0
            gv[:, 3] = 0
            return gc, gv, gx0, None

    return XPBDRollout


def __getattr__(name):
    if name == "XPBDRollout":
        fn = _autograd_function()
        globals()["XPBDRollout"] = fn
        return fn
    raise AttributeError(name)
