"""Reverse mode through the QG step: checkpointed adjoint runs and a
torch.autograd.Function over the C ABI's adjoint entry points.

The reference runs its model forward only; this module adds gradients of an
objective of the final state with respect to the initial stream function
and the Ekman-pumping forcing, for a closed box in FP64:

    run = AdjointRun(qg, every=20)     # checkpoint every 20 steps
    run.forward(nsteps, tdt)           # from the handle's current state
    g = run.backward(lp=dJ_dp)         # adjoint seeds of the final state
    g["gp0"], g["gpm0"], g["lwekp"]    # dJ/d(p, pm given to set_state), dJ/dwekp

forward() keeps a full-state slot at every `every`-th step (device memory).
backward() walks the segments last first: it reloads a segment's checkpoint,
recomputes the segment's steps keeping p and q of each step's input, then
reverses the steps last first (oqg_adj_segment queues all of it on the
handle's stream without host waits), so memory is
(nsteps/every) full states + `every` (p, q) pairs.  At the end the handle
holds the final state again.

`QGRun` wraps a whole run for autograd: psi0 (nl, nyp, nxp) FP64 and the
wind-stress curl field c (nyp, nxp), wekp = c / f0, to the final p.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from .core import QG, _check, lib


def _ptr(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(t.data_ptr())


def _dev_f64(x, shape, device):
    if x is None:
        return None
    t = torch.as_tensor(x, dtype=torch.float64, device=device).reshape(shape).contiguous()
    return t


class AdjointRun:
    def __init__(self, qg: QG, every: int = 20, device=None):
        if qg.b.cyclic or qg.b.precision != 0:
            raise ValueError("the adjoint covers the closed box in FP64 only")
        if every < 1:
            raise ValueError("every must be >= 1")
        self.qg = qg
        self.every = int(every)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        full, pq = ctypes.c_size_t(), ctypes.c_size_t()
        _check(lib().oqg_state_bytes(qg.h, ctypes.byref(full), ctypes.byref(pq)), "oqg_state_bytes")
        # slot rows rounded to 256 bytes
        self.full_bytes = (full.value + 255) // 256 * 256
        self.pq_bytes = (pq.value + 255) // 256 * 256
        self.ckpt = None
        self.slots = torch.empty((self.every, self.pq_bytes), dtype=torch.uint8, device=self.device)
        self.nsteps = 0

    def forward(self, nsteps: int, tdt: float) -> None:
        """Runs nsteps steps from the handle's current state, keeping a
        checkpoint before every `every`-th step."""
        qg = self.qg
        self.nsteps, self.tdt = int(nsteps), float(tdt)
        self.n0 = qg.step_index()
        nseg = (self.nsteps + self.every - 1) // self.every
        shape = (nseg + 1, self.full_bytes)
        if self.ckpt is None or tuple(self.ckpt.shape) != shape:
            self.ckpt = None   # release the old slots before making the new ones
            self.ckpt = torch.empty(shape, dtype=torch.uint8, device=self.device)
        torch.cuda.synchronize(self.device)
        for s in range(nseg):
            _check(lib().oqg_state_save(qg.h, _ptr(self.ckpt[s])), "oqg_state_save")
            qg.step(self.tdt, min(self.every, self.nsteps - s * self.every))
        _check(lib().oqg_state_save(qg.h, _ptr(self.ckpt[nseg])), "oqg_state_save")
        qg.sync()

    def backward(self, lp=None, lpm=None, lq=None, lqm=None, ldpi=None, ldpip=None):
        """Gradients of an objective J(final state) given its adjoint seeds
        (dJ/dp, dJ/dpm, dJ/dq, dJ/dqm as (nl, nyp, nxp), dJ/ddpi, dJ/ddpip).
        Returns torch FP64 tensors on the device: gp0, gpm0 (dJ with respect
        to the p and pm of set_state at the start), lwekp (dJ/dwekp, (nyp,
        nxp)), and the adjoint state at the start (lp, lpm, lq, lqm)."""
        qg, b = self.qg, self.qg.b
        if self.ckpt is None:
            raise RuntimeError("backward() needs a forward() first")
        L = lib()
        sh3 = b.shape3
        seeds = [_dev_f64(x, sh3, self.device) for x in (lp, lpm, lq, lqm)]
        d = lambda x: None if x is None else np.ascontiguousarray(x, dtype=np.float64).ctypes.data_as(
            ctypes.POINTER(ctypes.c_double))
        ldpi_a = None if ldpi is None else np.ascontiguousarray(ldpi, dtype=np.float64)
        ldpip_a = None if ldpip is None else np.ascontiguousarray(ldpip, dtype=np.float64)
        torch.cuda.synchronize(self.device)
        _check(L.oqg_adj_set(qg.h, *[None if t is None else _ptr(t) for t in seeds], d(ldpi_a), d(ldpip_a)),
               "oqg_adj_set")
        nseg = self.ckpt.shape[0] - 1
        for s in reversed(range(nseg)):
            n = min(self.every, self.nsteps - s * self.every)
            _check(L.oqg_adj_segment(qg.h, _ptr(self.ckpt[s]), _ptr(self.slots), ctypes.c_size_t(self.pq_bytes),
                                     n, ctypes.c_double(self.tdt),
                                     ctypes.c_longlong(self.n0 + s * self.every + 1)), "oqg_adj_segment")
        out = {k: torch.empty(sh3, dtype=torch.float64, device=self.device)
               for k in ("gp0", "gpm0", "lp", "lpm", "lq", "lqm")}
        out["lwekp"] = torch.empty(b.shape2, dtype=torch.float64, device=self.device)
        l1 = np.zeros(b.nl - 1)
        l2 = np.zeros(b.nl - 1)
        _check(L.oqg_adj_get(qg.h, _ptr(out["lp"]), _ptr(out["lpm"]), _ptr(out["lq"]), _ptr(out["lqm"]),
                             d(l1), d(l2), _ptr(out["lwekp"])), "oqg_adj_get")
        # oqg_adj_get's scalars come back through host arrays made above
        out["ldpi"], out["ldpip"] = l1, l2
        _check(L.oqg_adj_initial(qg.h, _ptr(out["gp0"]), _ptr(out["gpm0"])), "oqg_adj_initial")
        _check(L.oqg_state_load(qg.h, _ptr(self.ckpt[nseg])), "oqg_state_load")
        qg.sync()
        return out


def ekei(b, p: torch.Tensor, rho: float = 1.0e3) -> torch.Tensor:
    """Layer kinetic energies of qg_diagno (qg_monitor.F90:297-302, 331-333):
    0.5 rho h_k int (u^2 + v^2) dA with u = -dPdy_2bc(p)/f0, v = dPdx_2bc(p)/f0
    (numerics.F90:470-513), closed box; p (nl, nyp, nxp) torch FP64."""
    import torch.nn.functional as F
    ah = b.bcco * 0.5 + 1.0
    dx, dy = b.dx, b.dy
    vx = torch.cat([(p[..., :, 1:2] - p[..., :, 0:1]) / (dx * ah),
                    (p[..., :, 2:] - p[..., :, :-2]) / (2.0 * dx),
                    (p[..., :, -1:] - p[..., :, -2:-1]) / (dx * ah)], dim=-1)
    vx = F.pad(vx[..., 1:-1, :], (0, 0, 1, 1))
    uy = torch.cat([(p[..., 1:2, :] - p[..., 0:1, :]) / (dy * ah),
                    (p[..., 2:, :] - p[..., :-2, :]) / (2.0 * dy),
                    (p[..., -1:, :] - p[..., -2:-1, :]) / (dy * ah)], dim=-2)
    uy = F.pad(uy[..., :, 1:-1], (1, 1, 0, 0))
    wx = torch.ones(b.nxp, dtype=p.dtype, device=p.device)
    wy = torch.ones(b.nyp, dtype=p.dtype, device=p.device)
    wx[0] = wx[-1] = 0.5
    wy[0] = wy[-1] = 0.5
    w = wy[:, None] * wx[None, :] * (dx * dy)
    ke = ((uy / b.fnot) ** 2 + (vx / b.fnot) ** 2) * w
    h = torch.as_tensor(list(b.h), dtype=p.dtype, device=p.device)
    return 0.5 * rho * h * ke.sum(dim=(-2, -1))


class QGRun(torch.autograd.Function):
    """p_final = run(psi0, curl): set_state(f0 psi0, f0 psi0), forcing
    wekp = curl / f0, nsteps leapfrog steps of tdt from step index 0, and
    checkpoint-every-k recomputation on the way back."""

    @staticmethod
    def forward(ctx, psi0: torch.Tensor, curl: torch.Tensor, qg: QG, nsteps: int, tdt: float, every: int):
        b = qg.b
        f0 = b.fnot
        p0 = (f0 * psi0.detach().to(torch.float64)).reshape(b.shape3).cpu().numpy()
        wekp = (curl.detach().to(torch.float64) / f0).reshape(b.shape2).cpu().numpy()
        qg.set_state(p0, p0)
        qg.set_forcing(wekp, None, 0.0, 0.0)
        qg.set_step_index(0)
        run = AdjointRun(qg, every, device=psi0.device)
        run.forward(nsteps, tdt)
        ctx.run, ctx.f0, ctx.cdtype = run, f0, curl.dtype
        p = qg.get_state()[0]
        return torch.as_tensor(p, dtype=torch.float64, device=psi0.device)

    @staticmethod
    def backward(ctx, gp: torch.Tensor):
        g = ctx.run.backward(lp=gp.detach())
        gpsi = ctx.f0 * (g["gp0"] + g["gpm0"])
        gcurl = (g["lwekp"] / ctx.f0).to(ctx.cdtype)
        return gpsi, gcurl, None, None, None, None
