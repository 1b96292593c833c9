"""Plain-PyTorch FP64 restatement of one closed-box QG step, differentiable.

Test infrastructure: it is the autograd reference the hand-written adjoint is
checked against (a vector-Jacobian product of this step equals the adjoint
step's result to rounding).  It follows the same reference lines as the C++
oracle (oracle/oqg_oracle.cpp) for a closed box:

  step_qg                    src/qg/core.F90:16-33
  vort_step                  src/qg/vorticity.F90:14-103
  jacobian, del2_P_bc        src/glam/numerics.F90:340-388, 410-468
  solve_pressure             src/qg/pressure.F90:21-69
  p_modes_rhs, modes_to_layers  src/qg/modes.F90:248-284
  solve_inhomog_box          src/qg/inhomog.F90:170-212
  box_homog                  src/qg/homog.F90:331-366
  update_mass_constr         src/qg/constraint.F90:167-179
  ocqbdy                     src/qg/vorsubs.F90:58-114
  suppress_comp_mode         src/driver.F90:174-189
  qcomp, init_mass_constr    src/qg/vorsubs.F90:27-56, constraint.F90:145-165

The Helmholtz problems are solved with dense orthonormal sine bases in x and
y (the exact inverse of the reference's five-point operator with zero walls,
which the reference computes by a DST-I in x and Thomas solves in y).  The
init-time tables (vertical modes, the homogeneous solutions and their
constraint matrix) come from the oracle.  Fields are (nl, nyp, nxp) tensors.
"""
from __future__ import annotations

import math

import numpy as np
import torch
import torch.nn.functional as F


class TorchBox:
    def __init__(self, basin, oracle_handle, device="cpu"):
        b = basin
        if b.cyclic:
            raise ValueError("TorchBox restates the closed box only")
        self.b = b
        dt = torch.float64
        t = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64), dtype=dt, device=device)
        md = oracle_handle.modes()
        self.nl = b.nl
        self.amat = t(md["amat"])            # [k, l]
        self.ctl2m = t(md["ctl2m"])          # [k, m]
        self.ctm2l = t(md["ctm2l"])          # [m, k]
        self.rdm2 = t(md["rdm2"])
        self.hsb = t(oracle_handle.homog())  # (nl-1, nyp, nxp)
        nl = b.nl
        self.yprel = t(b.yprel)
        self.ah2 = t(b.ah2 if b.ah2 is not None else [0.0] * nl)
        self.ah4 = t(b.ah4 if b.ah4 is not None else [0.0] * nl)
        self.kt = b.ktopo() - 1
        self.ddyn = t(np.asarray(b.ddyn, dtype=np.float64).reshape(b.shape2)) if b.ddyn is not None else None
        f0 = b.fnot
        self.bcfac = b.bcco / (0.5 * b.bcco + 1.0)
        self.jac_fac = 1.0 / (3.0 * (2.0 * b.dx) * (2.0 * b.dy) * f0)
        fohfac = [f0 / h for h in b.h]
        self.c_wind = b.tau_sign * fohfac[0]
        self.c_drag = fohfac[self.kt] * b.delek / (2.0 * abs(f0))
        # trapezoid weights of int_P_dA
        wx = np.ones(b.nxp); wx[0] = wx[-1] = 0.5
        wy = np.ones(b.nyp); wy[0] = wy[-1] = 0.5
        self.w = t(np.outer(wy, wx) * b.dx * b.dy)
        # constraint matrix cdhoc (homog.F90:214-278)
        aipohs = (self.hsb * self.w).sum(dim=(1, 2))
        C = torch.zeros(nl - 1, nl - 1, dtype=dt, device=device)
        for k in range(nl - 1):
            for m in range(1, nl):
                C[k, m - 1] = (self.ctm2l[m, k + 1] - self.ctm2l[m, k]) * aipohs[m - 1]
        self.cdhoc = C
        # orthonormal sine bases and eigenvalues of the interior operator
        def sine(n, h):
            i = np.arange(1, n + 1)
            S = math.sqrt(2.0 / (n + 1)) * np.sin(np.pi * np.outer(i, i) / (n + 1))
            lam = (2.0 * np.cos(np.pi * i / (n + 1)) - 2.0) / (h * h)
            return t(S), t(lam)
        self.Sx, self.lx = sine(b.nxp - 2, b.dx)
        self.Sy, self.ly = sine(b.nyp - 2, b.dy)

    # -- stencils
    def lap(self, f):
        """del2_P_bc of every layer (numerics.F90:410-468)."""
        b = self.b
        fx, fy = 1.0 / (b.dx * b.dx), 1.0 / (b.dy * b.dy)
        c = self.bcfac
        X = torch.cat([c * (f[..., :, 1:2] - f[..., :, 0:1]),
                       f[..., :, :-2] + f[..., :, 2:] - 2.0 * f[..., :, 1:-1],
                       -c * (f[..., :, -1:] - f[..., :, -2:-1])], dim=-1) * fx
        X = F.pad(X[..., 1:-1, :], (0, 0, 1, 1))
        Y = torch.cat([c * (f[..., 1:2, :] - f[..., 0:1, :]),
                       f[..., :-2, :] + f[..., 2:, :] - 2.0 * f[..., 1:-1, :],
                       -c * (f[..., -1:, :] - f[..., -2:-1, :])], dim=-2) * fy
        Y = F.pad(Y[..., :, 1:-1], (1, 1, 0, 0))
        return X + Y

    @staticmethod
    def _dx2(f):   # dPdx_2, box (numerics.F90:311-325)
        return F.pad(f[..., :, 2:] - f[..., :, :-2], (1, 1, 0, 0))

    @staticmethod
    def _dy2(f):   # dPdy_2 (numerics.F90:327-338)
        return F.pad(f[..., 2:, :] - f[..., :-2, :], (0, 0, 1, 1))

    def jacobian(self, p, q):
        """jacobian(p, q) (numerics.F90:340-388), every layer."""
        dpx, dpy, dqx, dqy = self._dx2(p), self._dy2(p), self._dx2(q), self._dy2(q)
        t = (dqx * dpy - dqy * dpx + self._dx2(q * dpy) - self._dy2(q * dpx)
             + self._dy2(p * dqx) - self._dx2(p * dqy))
        return self.jac_fac * t

    def helmholtz(self, rhs):
        """solve_inhomog_box for every mode: (Del^2 - rdm2_m) u_m = rhs_m on the
        interior, u_m = 0 on the walls."""
        r = rhs[:, 1:-1, 1:-1]
        hat = self.Sy.T @ r @ self.Sx
        den = self.ly[None, :, None] + self.lx[None, None, :] - self.rdm2[:, None, None]
        u = self.Sy @ (hat / den) @ self.Sx.T
        return F.pad(u, (1, 1, 1, 1))

    def ocqbdy(self, p, q):
        """Wall values of q from p (vorsubs.F90:58-114): corners take the
        meridional-wall difference and the matmul, beta and topography terms
        twice, as the reference's loops do."""
        b = self.b
        fac = b.bcco / (b.dx * b.dx) / (0.5 * b.bcco + 1.0) / b.fnot
        nyp, nxp = b.nyp, b.nxp
        wall = torch.zeros(nyp, nxp, dtype=torch.bool, device=p.device)
        wall[0, :] = wall[-1, :] = wall[:, 0] = wall[:, -1] = True
        cnt = torch.zeros(nyp, nxp, dtype=p.dtype, device=p.device)
        cnt[0, :] += 1; cnt[-1, :] += 1; cnt[:, 0] += 1; cnt[:, -1] += 1
        nbr = torch.zeros_like(p)
        nbr = nbr + F.pad(p[:, 1:2, 1:-1] - p[:, 0:1, 1:-1], (1, 1, 0, nyp - 1))
        nbr = nbr + F.pad(p[:, -2:-1, 1:-1] - p[:, -1:, 1:-1], (1, 1, nyp - 1, 0))
        nbr = nbr + F.pad(p[:, :, 1:2] - p[:, :, 0:1], (0, nxp - 1, 0, 0))
        nbr = nbr + F.pad(p[:, :, -2:-1] - p[:, :, -1:], (nxp - 1, 0, 0, 0))
        Ap = torch.einsum("kl,lyx->kyx", self.amat, p)
        qw = fac * nbr - cnt * b.fnot * Ap + cnt * b.beta * self.yprel[None, :, None]
        if self.ddyn is not None:
            qw = qw + F.pad((cnt * self.ddyn)[None], (0, 0, 0, 0, self.kt, self.nl - 1 - self.kt))
        return torch.where(wall[None], qw, q)

    # -- the step
    def step(self, p, pm, q, qm, dpi, dpip, wekp, tdt, suppress=False):
        """One step_qg (ent = 0), then suppress_comp_mode when asked.  Returns
        (p, pm, q, qm, dpi, dpip) after the step."""
        b = self.b
        nl, kt = self.nl, self.kt
        dq = self.jacobian(p, q)
        d2 = self.lap(pm)
        d4 = self.lap(d2)
        d6 = self.lap(d4)
        dq = dq + self.ah2[:, None, None] / b.fnot * d4 - self.ah4[:, None, None] / b.fnot * d6
        add = [torch.zeros_like(wekp)] * nl
        add[0] = add[0] + self.c_wind * wekp
        add[kt] = add[kt] - self.c_drag * d2[kt]
        dq = dq + torch.stack(add)
        qn = qm + tdt * dq
        # solve_pressure
        ql = qn - b.beta * self.yprel[None, :, None]
        if self.ddyn is not None:
            ql = ql - F.pad(self.ddyn[None], (0, 0, 0, 0, kt, nl - 1 - kt))
        rhs = b.fnot * torch.einsum("km,kyx->myx", self.ctl2m, ql)
        inh = self.helmholtz(rhs)
        dpi_n, dpip_n = dpip, dpi
        im = (inh * self.w).sum(dim=(1, 2))
        ik = self.ctm2l.T @ im
        r = dpi_n - (ik[1:] - ik[:-1])
        alpha = torch.linalg.solve(self.cdhoc, r)
        hom = torch.cat([torch.zeros_like(inh[:1]), alpha[:, None, None] * self.hsb], dim=0)
        pn = torch.einsum("mk,myx->kyx", self.ctm2l, inh + hom)
        qn = self.ocqbdy(pn, qn)
        out = [pn, p, qn, q, dpi_n, dpip_n]
        if suppress:
            out[2] = 0.5 * (out[2] + out[3])
            out[0] = 0.5 * (out[0] + out[1])
            out[4] = 0.5 * (out[4] + out[5])
        return tuple(out)

    # -- init from (p, pm): set_state
    def qcomp(self, p):
        b = self.b
        q = self.lap(p) / b.fnot + b.beta * self.yprel[None, :, None]
        if self.ddyn is not None:
            q = q + F.pad(self.ddyn[None], (0, 0, 0, 0, self.kt, self.nl - 1 - self.kt))
        return q - b.fnot * torch.einsum("kl,lyx->kyx", self.amat, p)

    def mass(self, p):
        ip = (p * self.w).sum(dim=(1, 2))
        return self.b.dz_sign * (ip[:-1] - ip[1:])

    def init_state(self, p, pm):
        return p, pm, self.qcomp(p), self.qcomp(pm), self.mass(p), self.mass(pm)
