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
