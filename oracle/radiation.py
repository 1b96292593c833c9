"""CPU restatement of the radiation scheme's start-up (test infrastructure:
the checker of the library's host code, never the thing shipped).

Follows:
  load_rad, radiat and its helpers   src/mixed/radsubs.F90:63-674
  init_entrain_coeff                  src/mixed/amlsubs.F90:100-131
  init_temp_from_rad, zonal_temp      src/mixed/mixed.F90:102-151
  sin_lat                             src/glam/numerics.F90:516-525
with numpy arrays for the quadratures and numpy.linalg.solve for the
balance system.  The reference has no tests of this code: the restatement
is pinned by the balances its equations define (tests/test_radiation.py).
Indexes follow the Fortran ones: aup[k, l] is Aup(k, l), adown[k, l] is
Adown(k, l) (row 0 unused), dup[k] is Dup(k).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

STEFAN = 5.67040e-8
SIGOV2 = 0.5 * STEFAN
NZ = 10001


def trapin(f, delz):
    """The extended trapezoidal rule (radsubs.F90:661-674)."""
    return delz * (0.5 * f[0] + np.sum(f[1:-1]) + 0.5 * f[-1])


def bflux(t0, z, gamma):
    """B(T0, z, gamma) (radsubs.F90:338-344)."""
    return SIGOV2 * (t0 - z * gamma) ** 4


@dataclass
class RadState:
    fspco: float
    xlamda: float
    tauk: np.ndarray
    uprad: np.ndarray
    dnrad: np.ndarray
    uprad_m: float
    atm_tmbar: float
    ocn_tmbar: float
    fupbar: np.ndarray
    fdnbar: np.ndarray
    aup: np.ndarray
    adown: np.ndarray
    dup: np.ndarray
    d0up: float
    dmdown: float
    rbetat: np.ndarray
    rbtmat: float
    rbtmoc: float
    rbalar: np.ndarray


def radiat(h, hm, fnot, fsbar, fspamp, zopt, gamma, xlamda, tabsat):
    """load_rad + radiat for layer thicknesses h (nl), mixed-layer depth hm;
    zopt (nl+1) optical depths, tabsat (nl) absolute temperatures."""
    nl = len(h)
    zopt = np.asarray(zopt, dtype=np.float64)
    if fspamp < 0.0:
        raise ValueError("fspamp must be >= 0")
    fspco = float(np.copysign(abs(fspamp), fnot))
    tauk = np.empty(nl + 1)
    tauk[0] = np.exp(-hm / zopt[0])
    tauk[1] = np.exp(-(h[0] - hm) / zopt[1])
    for k in range(2, nl + 1):
        tauk[k] = np.exp(-h[k - 1] / zopt[k])
    uprad, dnrad = np.zeros(nl + 1), np.zeros(nl + 1)
    hbot, htop = hm, h[0]
    for k in range(1, nl + 1):
        if k > 1:
            hbot, htop = htop, htop + h[k - 1]
        delz = (htop - hbot) / (NZ - 1) if k == 1 else h[k - 1] / (NZ - 1)
        zz = hbot + np.arange(NZ) * delz
        T = tabsat[k - 1] - gamma * zz
        uprad[k] = trapin(SIGOV2 * T ** 4 * np.exp(-(htop - zz) / zopt[k]), delz) / zopt[k]
        dnrad[k] = trapin(SIGOV2 * T ** 4 * np.exp(-(zz - hbot) / zopt[k]), delz) / zopt[k]
    rhstat = 0.0
    for k in range(1, nl + 1):
        rhstat = rhstat * tauk[k] + uprad[k]
    rhstat = (-rhstat - fsbar) / np.prod(tauk[1:])
    atm = 300.0
    delz = hm / (NZ - 1)
    zz = np.arange(NZ) * delz
    for it in range(1, 400):
        uprad_m = trapin((atm - gamma * zz) ** 4 * np.exp(-(hm - zz) / zopt[0]), delz) * SIGOV2 / zopt[0]
        deltm = 0.25 * (rhstat - uprad_m) * atm / uprad_m
        atm = atm + 0.75 * deltm
        if abs(deltm) <= 1e-13:
            break
    else:
        raise RuntimeError("tmbara did not converge")
    rhstoc = xlamda * atm + bflux(atm, 0.0, 0.0) - fsbar
    ocn = atm
    for it in range(1, 400):
        told = ocn
        ocn = rhstoc / (xlamda + STEFAN * told ** 3)
        if abs(ocn - told) <= 1e-13:
            break
    else:
        raise RuntimeError("tmbaro did not converge")
    fupbar = np.zeros(nl + 1)
    fupbar[0] = uprad_m
    for k in range(1, nl + 1):
        fupbar[k] = fupbar[k - 1] * tauk[k] + uprad[k]
    fdnbar = np.zeros(nl + 2)
    fdnbar[nl] = -dnrad[nl]
    for k in range(nl - 1, 0, -1):
        fdnbar[k] = fdnbar[k + 1] * tauk[k] - dnrad[k]
    Z = np.zeros(nl + 1)
    Z[1:] = np.cumsum(h)
    btop, bbot = np.zeros(nl + 1), np.zeros(nl + 1)
    btop[0] = bflux(atm, hm, gamma)
    for k in range(1, nl + 1):
        btop[k] = bflux(tabsat[k - 1], Z[k], gamma)
    bbot[0] = bflux(atm, 0.0, gamma)
    bbot[1] = bflux(tabsat[0], hm, gamma)
    for k in range(2, nl + 1):
        bbot[k] = bflux(tabsat[k - 1], Z[k - 1], gamma)
    aup = np.zeros((nl + 1, nl))
    adown = np.zeros((nl + 1, nl))
    aup[0, 0] = (btop[0] - fupbar[0]) / zopt[0]
    for k in range(1, nl):
        aup[k, k] = (-tauk[k] * fupbar[k - 1] - uprad[k] + btop[k]) / zopt[k]
    for k in range(1, nl + 1):
        aup[k, k - 1] = tauk[k] * (aup[k - 1, k - 1] + fupbar[k - 1] / zopt[k] - bbot[k] / zopt[k])
    for k in range(2, nl + 1):
        for l in range(0, k - 1):
            aup[k, l] = aup[k - 1, l] * tauk[k]
    d0up = 4.0 * STEFAN * ocn ** 3
    dup = np.zeros(nl + 1)
    dup[0] = 2.0 * STEFAN * trapin((atm - gamma * zz) ** 3 * np.exp(-(hm - zz) / zopt[0]), delz) / zopt[0]
    for k in range(1, nl + 1):
        dup[k] = dup[k - 1] * tauk[k]
    for k in range(1, nl):
        adown[k, k - 1] = (fdnbar[k + 1] * tauk[k] - dnrad[k] + bbot[k]) / zopt[k]
    adown[nl, nl - 1] = (bbot[nl] - dnrad[nl]) / zopt[nl]
    for k in range(nl - 1, 0, -1):
        for l in range(k + 1, nl):
            adown[k, l] = adown[k + 1, l] * tauk[k]
        adown[k, k] = tauk[k] * (adown[k + 1, k] - fdnbar[k + 1] / zopt[k] - btop[k] / zopt[k])
    dmdown = -2.0 * STEFAN * atm ** 3
    rb = np.zeros((nl, nl))
    rb[0, :nl - 1] = adown[1, 1:nl]
    rb[0, nl - 1] = dup[0]
    for k in range(2, nl):
        rb[k - 1, :nl - 1] = adown[k + 1, 1:nl] + aup[k, 1:nl]
        rb[k - 1, nl - 1] = dup[k]
    rb[nl - 1, :nl - 1] = aup[nl, 1:nl]
    rb[nl - 1, nl - 1] = dup[nl]
    x = np.linalg.solve(rb, -np.ones(nl))
    rbtmat = float(x[nl - 1])
    rbtmoc = ((xlamda - dmdown) * rbtmat - 1.0) / (xlamda + d0up)
    return RadState(fspco, xlamda, tauk, uprad, dnrad, uprad_m, atm, ocn, fupbar, fdnbar, aup, adown, dup, d0up,
                    dmdown, x[:nl - 1].copy(), rbtmat, rbtmoc, rb)


def entrain_coeff(nl, rho_cp, dt_12, r: RadState):
    """init_entrain_coeff (amlsubs.F90:100-131): aface(1..nl-1), bface, dface."""
    rr = -1.0 / (rho_cp * dt_12)
    aface = np.array([rr * (0.0 + r.adown[1, l] - r.aup[nl, l]) for l in range(1, nl)])
    bface = rr * (r.aup[0, 0] + r.adown[1, 0] - r.aup[nl, 0])
    dface = rr * (r.dup[0] + 0.0 - r.dup[nl])
    return aface, bface, dface


def zonal_temp(nyt, y0, dy, fnot, ya0, yla, dt_ns):
    """zonal_temp / sin_lat (mixed.F90:144-151, numerics.F90:516-525) at the
    T rows of a basin with first p row y0, for the atmosphere's y range."""
    yc, yn = ya0 + 0.5 * yla, ya0 + yla
    y = (y0 + np.arange(nyt) * dy) + 0.5 * dy
    return -0.5 * np.copysign(abs(dt_ns), fnot) * np.sin((np.pi / 2.0) * (y - yc) / (yn - yc))
