"""The radiation scheme's start-up (load_rad, radiat, init_entrain_coeff,
zonal_temp; src/mixed/radsubs.F90:63-674, amlsubs.F90:100-182,
mixed.F90:102-151) through the library's host code (oqg_radiat,
oqg_entrain_coeff, oqg_zonal_temp): the coefficients the coupled forcing
(OceanMixedLayer.compute_forcing) and the mixed layers take."""
from __future__ import annotations

import ctypes

import numpy as np

from .core import _check, lib
from .params import OQG_MAX_NL, OqgRadParams, OqgRadState


def _bind(L):
    if getattr(L, "_rad_bound", False):
        return L
    vp = ctypes.c_void_p
    L.oqg_radiat.argtypes = [ctypes.c_int, vp, ctypes.c_double, ctypes.c_double, ctypes.POINTER(OqgRadParams),
                             ctypes.POINTER(OqgRadState)]
    L.oqg_entrain_coeff.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.POINTER(OqgRadState),
                                    vp, vp, vp]
    L.oqg_zonal_temp.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_double, vp]
    L._rad_bound = True
    return L


def radiat(h, hm: float, fnot: float, *, fsbar: float, fspamp: float, zopt, gamma: float, xlamda: float,
           tabsat) -> OqgRadState:
    """load_rad + radiat of an atmosphere with layer thicknesses h (nl) and
    mixed-layer depth hm; zopt has nl+1 optical depths (the mixed layer's
    first), tabsat the nl layers' absolute temperatures.  The result's `c`
    is the OqgRadCoeffs compute_forcing takes."""
    L = _bind(lib())
    nl = len(h)
    if len(zopt) != nl + 1 or len(tabsat) != nl:
        raise ValueError("zopt needs nl+1 values and tabsat nl")
    p = OqgRadParams(fsbar, fspamp, gamma, xlamda, (ctypes.c_double * (OQG_MAX_NL + 1))(*map(float, zopt)),
                     (ctypes.c_double * OQG_MAX_NL)(*map(float, tabsat)))
    hh = np.ascontiguousarray(h, dtype=np.float64)
    out = OqgRadState()
    _check(L.oqg_radiat(nl, hh.ctypes.data, float(hm), float(fnot), ctypes.byref(p), ctypes.byref(out)),
           "oqg_radiat")
    return out


def entrain_coeff(nl: int, rho_cp: float, dt_12: float, rad: OqgRadState):
    """init_entrain_coeff: (aface(1..nl-1), bface, dface) for the atmospheric
    mixed layer, rho_cp of air and dt_12 = T(1) - T(2)."""
    L = _bind(lib())
    aface = np.zeros(max(nl - 1, 1))
    b, d = ctypes.c_double(), ctypes.c_double()
    _check(L.oqg_entrain_coeff(nl, float(rho_cp), float(dt_12), ctypes.byref(rad), aface.ctypes.data,
                               ctypes.addressof(b), ctypes.addressof(d)), "oqg_entrain_coeff")
    return aface[:nl - 1].copy(), b.value, d.value


def zonal_temp(nyt: int, y0: float, dy: float, fnot: float, ya0: float, yla: float, dt_ns: float):
    """zonal_temp at the nyt T rows of a basin (first p row y0, spacing dy)
    for the atmosphere's y range [ya0, ya0 + yla]; dt_ns = |rbtm * fspco|."""
    L = _bind(lib())
    out = np.empty(nyt)
    _check(L.oqg_zonal_temp(int(nyt), float(y0), float(dy), float(fnot), float(ya0), float(yla), float(dt_ns),
                            out.ctypes.data), "oqg_zonal_temp")
    return out


def _ocean_profile(ba, bo, rad: OqgRadState):
    """zonal_temp of the ocean's temperature (init_temp_from_rad with rbtmoc)
    on its T rows; the ocean sits centred in the channel (load_grid)."""
    nyta, nyto = ba.nyp - 1, bo.nyp - 1
    nytoar = nyto // int(round(ba.dx / bo.dx))
    y0o = ((nyta - nytoar) // 2) * ba.dy
    return zonal_temp(nyto, y0o, bo.dy, bo.fnot, 0.0, nyta * ba.dy, abs(rad.rbtmoc * rad.c.fspco))


def coupled_start(ba, bo, *, hm_a: float, fsbar: float, fspamp: float, zopt, gamma: float, xlamda: float, tabsat,
                  rho_a: float, cp_a: float, t1_abs_o: float, t2_abs_o: float, rho_o: float, cp_o: float):
    """The coupled model's radiative start-up (openqg.F90:190-215): radiat on
    the atmosphere ba, then the mixed layers' temperature parameters
    (init_temp_from_rad), the atmosphere's entrainment coefficients and
    xc1ast (init_atmos_ml) and the ocean's wall temperatures (init_ocean_ml,
    omlsubs.F90:38-41).  The ocean bo sits at the channel's western end,
    centred in y (load_grid).  Returns (rad, atmos kwargs, ocean kwargs): the
    keyword arguments AtmosMixedLayer and OceanMixedLayer take for them."""
    rad = radiat(ba.h, hm_a, ba.fnot, fsbar=fsbar, fspamp=fspamp, zopt=zopt, gamma=gamma, xlamda=xlamda,
                 tabsat=tabsat)
    nl = ba.nl
    nyta, nyto = ba.nyp - 1, bo.nyp - 1
    yla = nyta * ba.dy
    dt12_a = tabsat[0] - tabsat[1]
    aface, bface, dface = entrain_coeff(nl, rho_a * cp_a, dt12_a, rad)
    xc = zonal_temp(nyta, 0.0, ba.dy, ba.fnot, 0.0, yla, abs(rad.rbtmat * rad.c.fspco))
    atm = dict(xc1ast=np.repeat(xc[:, None], ba.nxp - 1, axis=1), t1_rel=tabsat[0] - rad.atm_tmbar, dt_12=dt12_a,
               rho_cp=rho_a * cp_a, aface=tuple(aface), bface=bface, dface=dface)
    wall = _ocean_profile(ba, bo, rad)
    ocn = dict(t1_rel=t1_abs_o - rad.ocn_tmbar, dt_12=t1_abs_o - t2_abs_o, rho_cp=rho_o * cp_o,
               nval=float(wall[-1]), sval=float(wall[0]))
    return rad, atm, ocn


def rbal_states(ba, bo, rad: OqgRadState, atm: dict):
    """The radiative-balance initial states (init_dynamic_state with
    qg_state, oml_state and aml_state "rbal", openqg.F90:249-306): the
    atmosphere's pressure (nl, nyp, nxp), p_k = plfac_k fsprim(yprel) with
    plfac_1 = 0 and plfac_k = plfac_{k-1} - gp_{k-1} rbetat_{k-1}; the sst
    (nyt, nxt), zonal_temp on the ocean's rows; ast, the atmosphere's
    zonal_temp (its xc1ast, from coupled_start's atm).  p and pm, data and
    datam start equal."""
    nl, yla = ba.nl, (ba.nyp - 1) * ba.dy
    plfac = np.zeros(nl)
    for k in range(1, nl):
        plfac[k] = plfac[k - 1] - ba.gp[k - 1] * rad.rbetat[k - 1]
    yprel = -0.5 * yla + np.arange(ba.nyp) * ba.dy
    fsp = rad.c.fspco * 0.5 * np.sin(np.pi * yprel / yla)          # fsprim (radsubs.F90:97-114)
    p = plfac[:, None, None] * np.repeat(fsp[:, None], ba.nxp, axis=1)[None]
    sst = np.repeat(_ocean_profile(ba, bo, rad)[:, None], bo.nxp - 1, axis=1)
    return p, sst, atm["xc1ast"].copy()
