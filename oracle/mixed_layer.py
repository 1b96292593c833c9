"""CPU restatement of the ocean mixed-layer step and the Ekman fields that
feed it (test infrastructure: the checker of the device path, never the
thing measured or shipped).

Follows, for a closed box (the ocean):
  ekman_from_tau          src/coupler/ekman.F90:53-83
  step_oml                src/mixed/omlsubs.F90:69-119
  adv_diff, adv_vel       src/mixed/mixed_layer.F90:16-95
  del2_T, avg_T           src/glam/numerics.F90:109-163
  map_T_to_x_face / y_face, c_grid_advection, dPdx, dPdy, map_T_to_P
                          src/glam/numerics.F90:64-107, 223-309, 392-408
  init_mixed              src/mixed/mixed.F90:73-99 (state starts at init_val)
  compute_forcing, bilint src/mixed/forcing.F90:18-99, src/glam/numerics.F90:528-589

Arrays are numpy C-order views of the Fortran ones: a Fortran (nx, ny) array
is (ny, nx) here.  T-grid fields are (nyt, nxt) = (nyp-1, nxp-1).
The reference has no tests of this code; the restatement is checked by the
properties its equations imply (tests/test_mixed_layer.py) and its Ekman
part against the C++ oracle's ekman_from_tau.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def map_T_to_P(t):
    """numerics.F90:64-107, closed box: (nyt, nxt) -> (nyp, nxp)."""
    nyt, nxt = t.shape
    o = np.empty((nyt + 1, nxt + 1))
    o[1:-1, 1:-1] = 0.25 * (t[1:, 1:] + t[1:, :-1] + t[:-1, 1:] + t[:-1, :-1])
    o[0, 1:-1] = 0.5 * (t[0, :-1] + t[0, 1:])
    o[-1, 1:-1] = 0.5 * (t[-1, :-1] + t[-1, 1:])
    o[1:-1, 0] = 0.5 * (t[:-1, 0] + t[1:, 0])
    o[1:-1, -1] = 0.5 * (t[:-1, -1] + t[1:, -1])
    o[0, 0], o[0, -1], o[-1, 0], o[-1, -1] = t[0, 0], t[0, -1], t[-1, 0], t[-1, -1]
    return o


def ekman(taux, tauy, dx, dy, fnot, hm, tau_sign=1):
    """ekman_from_tau (ekman.F90:53-83), closed box: wind stress at p points
    (nyp, nxp) -> uek (nyt, nxp), vek (nyp, nxt), wekt (nyt, nxt), wekp (nyp, nxp)."""
    taux_t = 0.5 * (taux[:, 1:] + taux[:, :-1])          # map_P_to_x_face: (nyp, nxt)
    tauy_t = 0.5 * (tauy[1:, :] + tauy[:-1, :])          # map_P_to_y_face: (nyt, nxp)
    uek = (tau_sign / (fnot * hm)) * tauy_t
    vek = (-tau_sign / (fnot * hm)) * taux_t
    wekt = ((1.0 / (dx * fnot)) * (tauy_t[:, 1:] - tauy_t[:, :-1])
            - (1.0 / (dy * fnot)) * (taux_t[1:, :] - taux_t[:-1, :]))
    return uek, vek, wekt, map_T_to_P(wekt)


def del2_T(t, dx, north_flux, north_val, south_flux, south_val):
    """numerics.F90:109-145, closed box (no flux through the meridional walls)."""
    nyt, nxt = t.shape
    dt_x = np.zeros((nyt, nxt + 1))
    dt_x[:, 1:nxt] = t[:, 1:] - t[:, :-1]
    dt_y = np.zeros((nyt + 1, nxt))
    if south_flux:
        dt_y[0] = t[0] - south_val
    dt_y[1:nyt] = t[1:] - t[:-1]
    if north_flux:
        dt_y[nyt] = north_val - t[-1]
    return (1.0 / (dx * dx)) * (dt_x[:, 1:] - dt_x[:, :-1] + dt_y[1:] - dt_y[:-1])


@dataclass
class OmlParams:
    """The ocean mixed layer's parameters (init_ocean_ml, omlsubs.F90:27-67;
    temp_type, mixed.F90:28-44)."""
    hm: float = 100.0          # mixed-layer depth (m)
    rho_cp: float = 4.0e6      # rho * cp of sea water (J m^-3 K^-1)
    t1_rel: float = 10.0       # T_bar - T_(1) (K)
    dt_12: float = 5.0         # T(1) - T(2) (K)
    st2d: float = 1.0e3        # Laplacian SST diffusivity (m^2/s)
    st4d: float = 0.0          # biharmonic SST diffusivity (m^4/s)
    ycexp: float = 1.0         # geostrophic advection coefficient
    fluxn: bool = False        # heat-flux condition at the northern wall
    fluxs: bool = False        # heat-flux condition at the southern wall
    nval: float = 0.0          # boundary temperatures of those conditions (K)
    sval: float = 0.0


class OmlOracle:
    """The mixed layer of one closed basin: sst (data) and sstm (datam)."""

    def __init__(self, basin, prm: OmlParams, init_val: float = 0.0):
        self.b, self.prm = basin, prm
        nyt, nxt = basin.nyp - 1, basin.nxp - 1
        self.data = np.full((nyt, nxt), init_val)
        self.datam = np.full((nyt, nxt), init_val)

    def adv_diff(self, dp_dx, dp_dy, uek, vek):
        """mixed_layer.F90:16-58 with adv_vel (:60-95)."""
        b, m = self.b, self.prm
        t = self.data
        nyt, nxt = t.shape
        vel_u = (-m.ycexp / b.fnot) * dp_dy + uek           # (nyt, nxp)
        vel_u[:, 0] = 0.0
        vel_u[:, -1] = 0.0
        vel_v = (m.ycexp / b.fnot) * dp_dx + vek            # (nyp, nxt)
        vel_v[0] = vek[0] if m.fluxs else 0.0
        vel_v[-1] = vek[-1] if m.fluxn else 0.0
        mx = np.empty((nyt, nxt + 1))                       # map_T_to_x_face
        mx[:, 0] = t[:, 0]
        mx[:, 1:nxt] = 0.5 * (t[:, :-1] + t[:, 1:])
        mx[:, nxt] = t[:, -1]
        my = np.empty((nyt + 1, nxt))                       # map_T_to_y_face
        my[0] = t[0] if m.fluxs else 0.5 * (t[0] + m.sval)
        my[1:nyt] = 0.5 * (t[:-1] + t[1:])
        my[nyt] = t[-1] if m.fluxn else 0.5 * (t[-1] + m.nval)
        uT, vT = vel_u * mx, vel_v * my
        adv = (-1.0 / b.dx) * (uT[:, 1:] - uT[:, :-1]) + (-1.0 / b.dy) * (vT[1:] - vT[:-1])
        d2 = del2_T(self.datam, b.dx, m.fluxn, m.nval, m.fluxs, m.sval)
        d4 = del2_T(d2, b.dx, False, 0.0, False, 0.0)
        return adv + m.st2d * d2 - m.st4d * d4

    def step(self, p1, uek, vek, wekt, fnetoc, compute_ent, tdto, ent):
        """step_oml (omlsubs.F90:69-119): p1 (nyp, nxp) the QG layer-1
        pressure; ent (nl-1, nyp, nxp) is updated in place when compute_ent."""
        b, m = self.b, self.prm
        dp_dx = (1.0 / b.dx) * (p1[:, 1:] - p1[:, :-1])
        dp_dy = (1.0 / b.dy) * (p1[1:, :] - p1[:-1, :])
        half = 0.5 * wekt * (self.datam - m.t1_rel)
        sstnew = self.datam + tdto * (self.adv_diff(dp_dx, dp_dy, uek, vek)
                                      + (1.0 / (m.rho_cp * m.hm)) * fnetoc
                                      + (1.0 / m.hm) * (wekt * self.datam - half))
        dT_conv = np.maximum(0.0, m.t1_rel - sstnew)
        xfo = None
        if compute_ent:
            ent[:] = 0.0
            xfo = (-1.0 / m.dt_12) * half - (m.hm / (tdto * m.dt_12)) * dT_conv
            xfo = xfo - xfo.sum() / xfo.size
            ent[0] = map_T_to_P(xfo)
        self.datam = self.data.copy()
        self.data = sstnew + dT_conv
        return xfo


# ---------------------------------------------------------------- the channel
# The atmosphere's zonally periodic channel: the same equations with the
# cyclic branches of the numerics (column nxp-1 of a p field repeats column 0).

def map_T_to_P_cyclic(t):
    """numerics.F90:64-107, cyclic branches: (nyt, nxt) -> (nyp, nxp)."""
    nyt, nxt = t.shape
    o = np.empty((nyt + 1, nxt + 1))
    o[1:-1, 1:-1] = 0.25 * (t[1:, 1:] + t[1:, :-1] + t[:-1, 1:] + t[:-1, :-1])
    o[0, 1:-1] = 0.5 * (t[0, :-1] + t[0, 1:])
    o[-1, 1:-1] = 0.5 * (t[-1, :-1] + t[-1, 1:])
    o[1:-1, 0] = 0.25 * (t[1:, 0] + t[1:, -1] + t[:-1, 0] + t[:-1, -1])
    o[0, 0] = 0.5 * (t[0, 0] + t[0, -1])
    o[-1, 0] = 0.5 * (t[-1, 0] + t[-1, -1])
    o[:, -1] = o[:, 0]
    return o


def ekman_cyclic(taux, tauy, dx, dy, fnot, hm, tau_sign=-1):
    """ekman_from_tau (ekman.F90:53-83) for a channel: uek, vek, wekt, wekp
    and the boundary stress integrals txis, txin (:60-70)."""
    def int_P_dx(r):
        return (0.5 * r[0] + r[1:-1].sum() + 0.5 * r[-1]) * dx
    txis = 0.5 * int_P_dx(taux[0] + taux[1])
    txin = 0.5 * int_P_dx(taux[-2] + taux[-1])
    taux_t = 0.5 * (taux[:, 1:] + taux[:, :-1])
    tauy_t = 0.5 * (tauy[1:, :] + tauy[:-1, :])
    uek = (tau_sign / (fnot * hm)) * tauy_t
    vek = (-tau_sign / (fnot * hm)) * taux_t
    wekt = ((1.0 / (dx * fnot)) * (tauy_t[:, 1:] - tauy_t[:, :-1])
            - (1.0 / (dy * fnot)) * (taux_t[1:, :] - taux_t[:-1, :]))
    return uek, vek, wekt, map_T_to_P_cyclic(wekt), txis, txin


def del2_T_cyclic(t, dx, north_flux, north_val, south_flux, south_val):
    """numerics.F90:109-145, cyclic in x."""
    nyt, nxt = t.shape
    dt_x = np.empty((nyt, nxt + 1))
    dt_x[:, 1:nxt] = t[:, 1:] - t[:, :-1]
    dt_x[:, 0] = t[:, 0] - t[:, -1]
    dt_x[:, nxt] = dt_x[:, 0]
    dt_y = np.zeros((nyt + 1, nxt))
    if south_flux:
        dt_y[0] = t[0] - south_val
    dt_y[1:nyt] = t[1:] - t[:-1]
    if north_flux:
        dt_y[nyt] = north_val - t[-1]
    return (1.0 / (dx * dx)) * (dt_x[:, 1:] - dt_x[:, :-1] + dt_y[1:] - dt_y[:-1])


def adv_diff_cyclic(data, datam, dp_dx, dp_dy, uek, vek, fnot, dx, dy, d2, d4, ycexp, fluxn, fluxs, nval, sval):
    """mixed_layer.F90:16-95 in a channel (no wall in x, so vel_u is kept)."""
    t = data
    nyt, nxt = t.shape
    vel_u = (-ycexp / fnot) * dp_dy + uek
    vel_v = (ycexp / fnot) * dp_dx + vek
    vel_v[0] = vek[0] if fluxs else 0.0
    vel_v[-1] = vek[-1] if fluxn else 0.0
    mx = np.empty((nyt, nxt + 1))
    mx[:, 0] = 0.5 * (t[:, 0] + t[:, -1])
    mx[:, 1:nxt] = 0.5 * (t[:, :-1] + t[:, 1:])
    mx[:, nxt] = mx[:, 0]
    my = np.empty((nyt + 1, nxt))
    my[0] = t[0] if fluxs else 0.5 * (t[0] + sval)
    my[1:nyt] = 0.5 * (t[:-1] + t[1:])
    my[nyt] = t[-1] if fluxn else 0.5 * (t[-1] + nval)
    uT, vT = vel_u * mx, vel_v * my
    adv = (-1.0 / dx) * (uT[:, 1:] - uT[:, :-1]) + (-1.0 / dy) * (vT[1:] - vT[:-1])
    e2 = del2_T_cyclic(datam, dx, fluxn, nval, fluxs, sval)
    e4 = del2_T_cyclic(e2, dx, False, 0.0, False, 0.0)
    return adv + d2 * e2 - d4 * e4


@dataclass
class AmlParams:
    """The atmospheric mixed layer's parameters (init_atmos_ml,
    amlsubs.F90:61-98) and its entrainment coefficients (init_entrain_coeff,
    :100-131, which the radiation scheme provides)."""
    hm: float = 1000.0         # the box's mixed-layer depth (m)
    rho_cp: float = 1.0e3      # rho * cp of air (J m^-3 K^-1)
    t1_rel: float = -5.0       # T_bar - T_(1) (K)
    dt_12: float = 20.0        # T(1) - T(2) (K)
    hmamin: float = 100.0      # minimum mixed-layer height (m)
    hmadmp: float = 0.5        # mixed-layer height damping
    xcexp: float = 1.0         # entrainment coupling coefficient
    at2d: float = 2.5e4        # temperature diffusivities
    at4d: float = 0.0
    ahmd: float = 2.0e4        # height diffusivity
    aface: tuple = (0.0, 0.0)  # entrainment coefficients of eta(1..nl-1)
    bface: float = 0.0
    dface: float = 0.0


class AmlOracle:
    """The atmospheric mixed layer of a channel: ast and hmixa with their
    lagged values, xc1ast (set_xc1ast) and the topography dtop given."""

    def __init__(self, basin, prm: AmlParams, xc1ast, dtop):
        self.b, self.prm = basin, prm
        nyt, nxt = basin.nyp - 1, basin.nxp - 1
        self.ast = np.zeros((nyt, nxt))
        self.astm = np.zeros((nyt, nxt))
        self.hmx = np.full((nyt, nxt), prm.hm)
        self.hmxm = np.full((nyt, nxt), prm.hm)
        self.xc1ast = np.asarray(xc1ast, dtype=np.float64)
        self.dtop = np.asarray(dtop, dtype=np.float64)

    def step(self, p1, uek, vek, wekt, eta, fnetat, compute_ent, tdta, ent):
        """step_aml (amlsubs.F90:184-229) with compute_new_aml (:231-285) and
        compute_atmos_entrainment (:287-326)."""
        b, m = self.b, self.prm
        dp_dx = (1.0 / b.dx) * (p1[:, 1:] - p1[:, :-1])
        dp_dy = (1.0 / b.dy) * (p1[1:, :] - p1[:-1, :])
        tmrhs = adv_diff_cyclic(self.ast, self.astm, dp_dx, dp_dy, uek, vek, b.fnot, b.dx, b.dy,
                                m.at2d, m.at4d, 1.0, False, False, 0.0, 0.0)
        dhdt = adv_diff_cyclic(self.hmx, self.hmxm, dp_dx, dp_dy, uek, vek, b.fnot, b.dx, b.dy,
                               m.ahmd, 0.0, 1.0, True, True, m.hm, m.hm)
        dT = m.t1_rel - self.astm
        hdrcdt = m.hmadmp / m.rho_cp
        hnew = np.full(dT.shape, m.hm)
        dT_fix = np.zeros(dT.shape)
        act = dT >= 2.0 * hdrcdt * tdta
        with np.errstate(divide="ignore", invalid="ignore"):
            diab = hdrcdt * (self.hmxm - m.hm) / dT
            hn = self.hmxm + tdta * (dhdt - diab)
            fix = np.maximum(m.hmamin - hn, 0.0)
            hn = hn + fix
            dfix = fix * dT / self.hmxm
        hnew[act] = hn[act]
        dT_fix[act] = dfix[act]
        tmrhs = tmrhs + (1.0 / m.rho_cp) * fnetat / self.hmxm - (1.0 / m.hm) * wekt * self.astm
        astnew = self.astm + tdta * tmrhs + dT_fix
        dT_conv = np.minimum(0.0, m.t1_rel - astnew)
        astnew = astnew + dT_conv
        if compute_ent:
            xfa = (m.xcexp * m.bface * (self.hmxm - m.hm)
                   + m.dface * (m.xcexp * self.astm + (1.0 - m.xcexp) * self.xc1ast)
                   + (m.xcexp / (tdta * m.dt_12)) * self.hmx * dT_conv)
            ent[:] = 0.0
            e1 = map_T_to_P_cyclic(xfa)
            for k in range(b.nl - 1):
                e1 = e1 + m.aface[k] * eta[k]
            ent[0] = e1 + m.bface * self.dtop
        self.astm, self.ast = self.ast, astnew
        self.hmxm, self.hmx = self.hmx, hnew


def atmos_stress(pm1, basin, cdat, hm):
    """The atmosphere's wind stress from its lagged layer-1 pressure (xforc,
    windstress.F90:102-148, without the ocean-velocity dependence), with
    dPdx_2bc / dPdy_2bc (numerics.F90:470-513) of a channel; pm1 (nyp, nxp)."""
    b = basin
    ah = 0.5 * b.bcco + 1.0
    dpdx = np.zeros_like(pm1)
    dpdx[:, 1:-1] = (pm1[:, 2:] - pm1[:, :-2]) / (2.0 * b.dx)
    dpdx[:, 0] = (pm1[:, 1] - pm1[:, -2]) / (2.0 * b.dx)
    dpdx[:, -1] = dpdx[:, 0]
    dpdx[0] = 0.0
    dpdx[-1] = 0.0
    dpdy = np.empty_like(pm1)
    dpdy[1:-1] = (pm1[2:] - pm1[:-2]) / (2.0 * b.dy)
    dpdy[0] = (pm1[1] - pm1[0]) / (b.dy * ah)
    dpdy[-1] = (pm1[-1] - pm1[-2]) / (b.dy * ah)
    u, v = -dpdy / b.fnot, dpdx / b.fnot
    cdhfaa = (cdat / b.fnot) / hm
    qpreaa = 1.0 / (abs(cdhfaa) * np.sqrt(2.0))
    u2 = 4.0 * cdhfaa * cdhfaa * (u * u + v * v)
    shrmag = qpreaa * np.sqrt(-1.0 + np.sqrt(1.0 + u2))
    cuohf = cdhfaa * shrmag
    cdochi = cdat * shrmag / (1.0 + cuohf * cuohf)
    return cdochi * (u - cuohf * v), cdochi * (v + cuohf * u)


# ------------------------------------------------------- stress on the ocean
def _dx_bc_c(f, dx):
    """dPdx_2bc of a channel field (numerics.F90:470-492)."""
    o = np.zeros_like(f)
    o[:, 1:-1] = (f[:, 2:] - f[:, :-2]) / (2.0 * dx)
    o[:, 0] = (f[:, 1] - f[:, -2]) / (2.0 * dx)
    o[:, -1] = o[:, 0]
    o[0] = 0.0
    o[-1] = 0.0
    return o


def _dy_bc_c(f, dy, ah):
    """dPdy_2bc of a channel field (numerics.F90:494-513)."""
    o = np.empty_like(f)
    o[1:-1] = (f[2:] - f[:-2]) / (2.0 * dy)
    o[0] = (f[1] - f[0]) / (dy * ah)
    o[-1] = (f[-1] - f[-2]) / (dy * ah)
    return o


def _dxx_bc_c(f, dx):
    """dP2dx2_bc of a channel field (numerics.F90:427-448)."""
    fac = 1.0 / (dx * dx)
    o = np.zeros_like(f)
    o[:, 1:-1] = fac * (f[:, :-2] + f[:, 2:] - 2.0 * f[:, 1:-1])
    o[:, 0] = fac * (f[:, -2] + f[:, 1] - 2.0 * f[:, 0])
    o[:, -1] = o[:, 0]
    o[0] = 0.0
    o[-1] = 0.0
    return o


def _dyy_bc_c(f, dy, alpha):
    """dP2dy2_bc of a channel field (numerics.F90:450-468)."""
    fac = 1.0 / (dy * dy)
    o = np.empty_like(f)
    o[1:-1] = fac * (f[:-2] + f[2:] - 2.0 * f[1:-1])
    o[0] = fac * alpha / (0.5 * alpha + 1.0) * (f[1] - f[0])
    o[-1] = -fac * alpha / (0.5 * alpha + 1.0) * (f[-1] - f[-2])
    return o


def coupling_grid(bo, ba):
    """load_grid (grid.F90:36-59): the atmosphere/ocean resolution ratio
    ndxr, the ocean's cells at atmospheric resolution and the 0-based first
    atmospheric p row and column of the ocean."""
    ndxr = int(round(ba.dx / bo.dx))
    nxtoar, nytoar = (bo.nxp - 1) // ndxr, (bo.nyp - 1) // ndxr
    ny1 = (ba.nyp - 1 - nytoar) // 2
    return ndxr, nxtoar, nytoar, 0, ny1


def hermite_bicubic(f, fx, fy, fxy, ndxr):
    """Bicubic interpolation of nodal values and scaled derivatives (per unit
    cell: fx = dx df/dx, ...) on (n+1, m+1) nodes to the ndxr-times finer
    grid; the interpolant is the tensor product of the cubic Hermite bases,
    the unique bicubic matching the 16 values of each cell (the role of
    new_bicubic, bicubic.F90:24-85).  Shared cell edges take the later cell,
    as bc3 writes them."""
    ny, nx = f.shape[0] - 1, f.shape[1] - 1
    io = np.arange(nx * ndxr + 1)
    jo = np.arange(ny * ndxr + 1)
    ci = np.minimum(io // ndxr, nx - 1)
    cj = np.minimum(jo // ndxr, ny - 1)
    s = (io - ci * ndxr) / ndxr
    t = (jo - cj * ndxr) / ndxr
    H0 = lambda x: 1.0 - 3.0 * x * x + 2.0 * x * x * x
    H1 = lambda x: 3.0 * x * x - 2.0 * x * x * x
    K0 = lambda x: x - 2.0 * x * x + x * x * x
    K1 = lambda x: -x * x + x * x * x
    out = np.zeros((jo.size, io.size))
    S, T = s[None, :], t[:, None]
    for a, (Ha, Ka) in enumerate(((H0, K0), (H1, K1))):
        for c, (Hc, Kc) in enumerate(((H0, K0), (H1, K1))):
            J, I = (cj + c)[:, None], (ci + a)[None, :]
            out = out + (f[J, I] * Ha(S) * Hc(T) + fx[J, I] * Ka(S) * Hc(T)
                         + fy[J, I] * Ha(S) * Kc(T) + fxy[J, I] * Ka(S) * Kc(T))
    return out


def _dx_bc_box(f, dx, alpha):
    """dPdx_2bc of a closed-box field (numerics.F90:470-492)."""
    o = np.empty_like(f)
    o[:, 1:-1] = (f[:, 2:] - f[:, :-2]) / (2.0 * dx)
    o[:, 0] = (f[:, 1] - f[:, 0]) / (dx * (0.5 * alpha + 1.0))
    o[:, -1] = (f[:, -1] - f[:, -2]) / (dx * (0.5 * alpha + 1.0))
    o[0] = 0.0
    o[-1] = 0.0
    return o


def _dy_bc_box(f, dy, alpha):
    """dPdy_2bc of a closed-box field (numerics.F90:494-513)."""
    o = np.empty_like(f)
    o[1:-1] = (f[2:] - f[:-2]) / (2.0 * dy)
    o[0] = (f[1] - f[0]) / (dy * (0.5 * alpha + 1.0))
    o[-1] = (f[-1] - f[-2]) / (dy * (0.5 * alpha + 1.0))
    o[:, 0] = 0.0
    o[:, -1] = 0.0
    return o


def ocean_stress(pma1, ba, bo, cdat, hma, raoro, pmo1=None, hmo=None, atmos_tau=None):
    """The ocean's wind stress from the atmosphere's lagged layer-1 pressure
    (compute_windstress, atmos_geos_vel, atmos_windstress; windstress.F90:
    150-314): the atmospheric geostrophic velocity and its derivatives on the
    atmospheric p points over the ocean, interpolated bicubically to the
    ocean's p points, the drag law there, times the density ratio raoro.
    Returns taux, tauy (nyp, nxp).  Given the ocean's lagged layer-1 pressure
    pmo1 and mixed-layer depth hmo (tau_udiff, :255-276), the velocity is the
    difference with the ocean's, and atmos_tau = (taux_a, tauy_a), if given,
    takes the ocean-resolution stress at the shared p points (:179-187)."""
    ndxr, nxtoar, nytoar, c0, r0 = coupling_grid(bo, ba)
    ah = 0.5 * ba.bcco + 1.0
    p = pma1
    dpdx, dpdy = _dx_bc_c(p, ba.dx), _dy_bc_c(p, ba.dy, ah)
    d2x, d2y = _dxx_bc_c(p, ba.dx), _dyy_bc_c(p, ba.dy, ba.bcco)
    dxy = _dx_bc_c(dpdy, ba.dx)
    dxxy, dxyy = _dx_bc_c(dxy, ba.dx), _dx_bc_c(d2y, ba.dx)
    sub = (slice(r0, r0 + nytoar + 1), slice(c0, c0 + nxtoar + 1))
    f0, dx, dy = ba.fnot, ba.dx, ba.dy
    u = hermite_bicubic(-dpdy[sub] / f0, -(dx / f0) * dxy[sub], -(dy / f0) * d2y[sub],
                        -(dx * dy / f0) * dxyy[sub], ndxr)
    v = hermite_bicubic(dpdx[sub] / f0, (dx / f0) * d2x[sub], (dy / f0) * dxy[sub],
                        (dx * dy / f0) * dxxy[sub], ndxr)
    if pmo1 is not None:
        u = u + _dy_bc_box(pmo1, bo.dy, bo.bcco) / bo.fnot
        v = v - _dx_bc_box(pmo1, bo.dx, bo.bcco) / bo.fnot
        cdhfaa = (cdat / f0) * (1.0 / hma + raoro / hmo)
    else:
        cdhfaa = (cdat / f0) / hma
    qpreaa = 1.0 / (abs(cdhfaa) * np.sqrt(2.0))
    shrmag = np.sqrt(-1.0 + np.sqrt(1.0 + 4.0 * cdhfaa * cdhfaa * (u * u + v * v)))
    cuohf = (qpreaa * cdhfaa) * shrmag
    cdchi = (qpreaa * cdat) * shrmag / (1.0 + cuohf * cuohf)
    tx, ty = cdchi * (u - cuohf * v), cdchi * (v + cuohf * u)
    if pmo1 is not None and atmos_tau is not None:
        for a, t in zip(atmos_tau, (tx, ty)):
            a[r0:r0 + nytoar + 1, c0:c0 + nxtoar + 1] = t[::ndxr, ::ndxr]
    return raoro * tx, raoro * ty


# ------------------------------------------------------------ coupled fluxes
@dataclass
class RadCoeffs:
    """The radiation coefficients compute_forcing reads (radiate_type,
    radsubs.F90:15-54), the derived values radiat computes at start-up."""
    fspco: float
    xlamda: float
    d0up: float
    dmdown: float
    dup0: float
    aup00: float
    adown10: float
    adown11: float


def bilint(at, bo, ba):
    """bilint (numerics.F90:528-589): the atmospheric T field at (nyt_a,
    nxt_a) interpolated bilinearly to the ocean's T points.  The ocean's
    origin is the atmospheric cell of coupling_grid; x is cyclic, and the
    first and last T rows hold beyond the channel's ends.  Indexes stay
    1-based and truncate like Fortran's int, as there."""
    _, _, _, c0, r0 = coupling_grid(bo, ba)
    nxta, nyta = ba.nxp - 1, ba.nyp - 1
    nxto, nyto = bo.nxp - 1, bo.nyp - 1
    dxainv, dyainv = 1.0 / ba.dx, 1.0 / ba.dy
    xta1, yta1 = 0.5 * ba.dx, 0.5 * ba.dy
    io = np.arange(nxto)
    xto = (c0 * ba.dx + io * bo.dx) + 0.5 * bo.dx
    iam = np.trunc(1.0 + dxainv * (xto - xta1)).astype(np.int64)
    iap = iam + 1
    xam = np.where(iam >= 1, (iam - 1) * ba.dx + xta1, xta1 - ba.dx)
    wpx = dxainv * (xto - xam)
    wmx = 1.0 - wpx
    iam = 1 + np.mod(iam + nxta - 1, nxta)
    iap = 1 + np.mod(iap + nxta - 1, nxta)
    out = np.empty((nyto, nxto))
    for jo in range(nyto):
        yto = (r0 * ba.dy + jo * bo.dy) + 0.5 * bo.dy
        jam = int(np.trunc(1.0 + dyainv * (yto - yta1)))
        jap = jam + 1
        jam = min(max(jam, 1), nyta)
        jap = min(jap, nyta)
        wpy = dyainv * (yto - ((jam - 1) * ba.dy + yta1))
        wmy = 1.0 - wpy
        rm, rp = at[jam - 1], at[jap - 1]
        out[jo] = (wmx * wmy * rm[iam - 1] + wpx * wmy * rm[iap - 1]
                   + wmx * wpy * rp[iam - 1] + wpx * wpy * rp[iap - 1])
    return out


def fsprim(fspco, yrel, yla):
    """The perturbative radiative forcing (fsprim, radsubs.F90:97-114)."""
    return fspco * 0.5 * np.sin(np.pi * yrel / yla)


def compute_forcing(sstm, astm, hmxm, pma, ba, bo, rad: RadCoeffs, hma, hmadmp, dtop=None):
    """compute_forcing (forcing.F90:18-99): the ocean's net flux fnetoc
    (nyt_o, nxt_o) and the atmosphere's fnetat (nyt_a, nxt_a) from the lagged
    sst, the atmosphere's lagged temperature astm and height hmxm, its lagged
    pressure pma (nl, nyp, nxp) for eta_1 = (pm_1 - pm_2) / gp_1, and its
    topography dtop (nyp, nxp) or None (flat)."""
    ndxr, nxtoar, nytoar, c0, r0 = coupling_grid(bo, ba)
    nxta, nyta = ba.nxp - 1, ba.nyp - 1
    nxto, nyto = bo.nxp - 1, bo.nyp - 1
    yla, ylo = nyta * ba.dy, nyto * bo.dy
    asto = bilint(astm, bo, ba)
    ocn_ir_up = rad.d0up * sstm
    sense_lat = rad.xlamda * (sstm - asto)
    aml_ir_down = rad.dmdown * asto
    yta = (-0.5 * yla + np.arange(nyta) * ba.dy) + 0.5 * ba.dy
    fnetat = -rad.dup0 * astm - fsprim(rad.fspco, yta, yla)[:, None]
    over = (slice(r0, r0 + nytoar), slice(c0, c0 + nxtoar))
    fnetat[over] = fnetat[over] + (rad.dmdown - rad.dup0) * astm[over]
    yto = (-0.5 * ylo + np.arange(nyto) * bo.dy) + 0.5 * bo.dy
    fsp = fsprim(rad.fspco, yto, yla)[:, None]
    fnetoc = -fsp - aml_ir_down - ocn_ir_up - sense_lat
    ocfrac = bo.dx * bo.dy / (ba.dx * ba.dy)
    up = ocn_ir_up + sense_lat
    for jo in range(nyto):
        ja = r0 + jo // ndxr
        for io in range(nxto):
            ia = c0 + io // ndxr
            fnetat[ja, ia] = fnetat[ja, ia] + ocfrac * up[jo, io]
    eta = (pma[0] - pma[1]) / ba.gp[0]
    p2t = lambda f, fac: (fac * 0.25) * (f[:-1, :-1] + f[:-1, 1:] + f[1:, :-1] + f[1:, 1:])
    fmafac = rad.adown11
    fmatop = rad.aup00 + rad.adown10
    hmafac = -hmadmp - rad.aup00 - rad.adown10
    top = p2t(dtop, fmatop) if dtop is not None else 0.0
    fnetat = fnetat - p2t(eta, fmafac) - top + hmafac * (hmxm - hma)
    return fnetoc, fnetat
