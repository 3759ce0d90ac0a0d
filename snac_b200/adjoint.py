"""FP64 adjoint of the SNAC step through the C ABI (snac_gpu_adjoint).

    loss, g = adjoint(ctx, nsteps, target_vy, target_y)   # g["cohesion"], g["friction"], g["viscosity"]
    r = adjoint(ctx, nsteps, target_vy, target_y, state=True)
    # also r.grad["coordinates"], ["velocity"] ([nn, 3]), ["stress"] ([ne*10, 6]),
    # ["plastic_strain"] ([ne*10]): gradients with respect to the entry state
    # (snac_gpu_adjoint_grads)

`SnacMisfit` wraps the same call as a torch.autograd.Function of the three
per-element scale fields:

    coh = torch.ones(ne, dtype=torch.float64, requires_grad=True)
    L = SnacMisfit.apply(coh, fric, visc, make_cfg, nsteps, target_vy, target_y)
    L.backward()          # coh.grad = dL/d(cohesion scale), ...

The loss is L = sum over the top-surface nodes of
w_v (v_y - target_vy)^2 + w_h (y - target_y)^2 after nsteps steps; the
checkpointed forward and the reverse sweep run on the GPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Dict, Optional, Tuple

import numpy as np

from .abi import SnacConfig, State
from .context import SnacContext, load_library

_DP = C.POINTER(C.c_double)


class AdjointDesc(C.Structure):
    _fields_ = [("nsteps", C.c_int), ("checkpoint_every", C.c_int), ("target_vy", _DP), ("target_y", _DP),
                ("w_v", C.c_double), ("w_h", C.c_double)]


class AdjointGrads(C.Structure):
    _fields_ = [(k, _DP) for k in ("cohesion", "friction", "viscosity", "coordinates", "velocity", "stress",
                                   "plastic_strain")]


class AdjointStats(C.Structure):
    _fields_ = [("ms_forward", C.c_double), ("ms_reverse", C.c_double), ("checkpoint_every", C.c_int),
                ("checkpoints", C.c_int)]


def _bind():
    lib = load_library()
    if not getattr(lib, "_adjoint_bound", False):
        lib.snac_gpu_adjoint.argtypes = [C.c_void_p, C.POINTER(AdjointDesc), _DP, _DP, _DP, _DP,
                                         C.POINTER(AdjointStats)]
        lib.snac_gpu_adjoint.restype = C.c_int
        lib.snac_gpu_adjoint_grads.argtypes = [C.c_void_p, C.POINTER(AdjointDesc), _DP, C.POINTER(AdjointGrads),
                                               C.POINTER(AdjointStats)]
        lib.snac_gpu_adjoint_grads.restype = C.c_int
        lib.snac_gpu_misfit.argtypes = [C.c_void_p, C.POINTER(AdjointDesc), _DP]
        lib.snac_gpu_misfit.restype = C.c_int
        lib._adjoint_bound = True
    return lib


def top_surface(cfg: SnacConfig, s: State) -> Tuple[np.ndarray, np.ndarray]:
    """(v_y, y) of the top node plane (j = ny) in node order i + k (nx + 1)."""
    nnx, nny, nnz = cfg.nx + 1, cfg.ny + 1, cfg.nz + 1
    v = s.velocity.reshape(nnz, nny, nnx, 3)[:, nny - 1, :, 1].reshape(-1)
    y = s.coord.reshape(nnz, nny, nnx, 3)[:, nny - 1, :, 1].reshape(-1)
    return np.ascontiguousarray(v), np.ascontiguousarray(y)


def _desc(nsteps, target_vy, target_y, w_v, w_h, checkpoint_every):
    tv = np.ascontiguousarray(target_vy, dtype=np.float64)
    ty = np.ascontiguousarray(target_y, dtype=np.float64)
    d = AdjointDesc(int(nsteps), int(checkpoint_every), tv.ctypes.data_as(_DP), ty.ctypes.data_as(_DP),
                    float(w_v), float(w_h))
    return d, (tv, ty)


@dataclass
class AdjointResult:
    loss: float
    grad: Dict[str, np.ndarray]
    ms_forward: float
    ms_reverse: float
    checkpoint_every: int
    checkpoints: int


def adjoint(ctx: SnacContext, nsteps: int, target_vy, target_y, w_v: float = 1.0, w_h: float = 1.0,
            checkpoint_every: int = 0, state: bool = False) -> AdjointResult:
    """Loss after nsteps steps from the context's current state and its
    gradient with respect to the per-element cohesion, friction and viscosity
    scales, and with state=True also with respect to the entry state
    (coordinates, velocities, tet stresses and plastic strains).  The context
    ends at the forward's final state."""
    lib = _bind()
    d, keep = _desc(nsteps, target_vy, target_y, w_v, w_h, checkpoint_every)
    ne, nn, nq = ctx.ne, ctx.nn, ctx.ne * 10
    g = {k: np.zeros(ne) for k in ("cohesion", "friction", "viscosity")}
    if state:
        g.update(coordinates=np.zeros((nn, 3)), velocity=np.zeros((nn, 3)), stress=np.zeros((nq, 6)),
                 plastic_strain=np.zeros(nq))
    gr = AdjointGrads(**{k: v.ctypes.data_as(_DP) for k, v in g.items()})
    loss = C.c_double()
    st = AdjointStats()
    rc = lib.snac_gpu_adjoint_grads(ctx.h, C.byref(d), C.byref(loss), C.byref(gr), C.byref(st))
    ctx._check(rc)
    return AdjointResult(loss.value, g, st.ms_forward, st.ms_reverse, st.checkpoint_every, st.checkpoints)


def misfit(ctx: SnacContext, target_vy, target_y, w_v: float = 1.0, w_h: float = 1.0) -> float:
    """The loss of the context's current state."""
    lib = _bind()
    d, keep = _desc(1, target_vy, target_y, w_v, w_h, 0)
    loss = C.c_double()
    ctx._check(lib.snac_gpu_misfit(ctx.h, C.byref(d), C.byref(loss)))
    return loss.value


def forward_loss(make_cfg: Callable[[np.ndarray, np.ndarray, np.ndarray], SnacConfig], coh, fric, visc,
                 nsteps: int, target_vy, target_y, w_v: float = 1.0, w_h: float = 1.0) -> float:
    """Loss of a plain forward run (no adjoint), for finite differences."""
    with SnacContext(make_cfg(coh, fric, visc)) as ctx:
        ctx.time_step_zero()
        ctx.step(nsteps)
        return misfit(ctx, target_vy, target_y, w_v, w_h)


try:
    import torch

    class SnacMisfit(torch.autograd.Function):
        """L(cohesion scale, friction scale, viscosity scale) with its FP64 adjoint."""

        @staticmethod
        def forward(ctx, coh, fric, visc, make_cfg, nsteps, target_vy, target_y, w_v=1.0, w_h=1.0,
                    checkpoint_every=0):
            cfg = make_cfg(coh.detach().cpu().numpy(), fric.detach().cpu().numpy(), visc.detach().cpu().numpy())
            with SnacContext(cfg) as m:
                m.time_step_zero()
                r = adjoint(m, nsteps, target_vy, target_y, w_v, w_h, checkpoint_every)
            ctx.save_for_backward(*(torch.from_numpy(r.grad[k]).to(coh.device) for k in ("cohesion", "friction",
                                                                                         "viscosity")))
            return torch.tensor(r.loss, dtype=torch.float64, device=coh.device)

        @staticmethod
        def backward(ctx, gout):
            gc, gf, gv = ctx.saved_tensors
            return gout * gc, gout * gf, gout * gv, None, None, None, None, None, None, None
except ImportError:  # torch is optional for the plain ctypes API
    SnacMisfit = None
