"""The radiation scheme's start-up (oqg_radiat, oqg_entrain_coeff,
oqg_zonal_temp; host code of the library, no device) against the numpy
restatement (oracle/radiation.py), and the restatement pinned by the
balances its equations define: the top-of-atmosphere balance of the mean
state, the ocean surface balance, the exact integrals of an isothermal
layer, and the residual of the balance system.

Parameters: the reference's atmosphere configuration (data/basin/atm_dg.cdl:
hm 1000 m, h 2000/3000/4000 m, T_abs 330/340/350 K, fsbar -210, fspamp 80,
zopt 200 / 3e4 / 3e4 / 4e4 m, gamma 1e-2 K/m, xlamda 35), and variants.
Tolerance: 1e-12 relative (the same FP64 arithmetic, sums in a different
order)."""
import numpy as np
import pytest

from oracle import radiation as R
from openqg_b200.core import OqgError
from openqg_b200.radiation import entrain_coeff, radiat, zonal_temp

DG = dict(h=[2000.0, 3000.0, 4000.0], hm=1000.0, fsbar=-210.0, fspamp=80.0, zopt=[200.0, 3.0e4, 3.0e4, 4.0e4],
          gamma=1.0e-2, xlamda=35.0, tabsat=[330.0, 340.0, 350.0])
TWO = dict(h=[3000.0, 6000.0], hm=800.0, fsbar=-220.0, fspamp=60.0, zopt=[250.0, 2.5e4, 4.0e4], gamma=8.0e-3,
           xlamda=30.0, tabsat=[320.0, 335.0])


def _close(a, b, tol=1e-12):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return np.max(np.abs(a - b)) <= tol * max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("cfg,fnot", [(DG, 1.0e-4), (DG, -1.0e-4), (TWO, 1.0e-4)])
def test_radiat_matches_oracle(cfg, fnot):
    nl = len(cfg["h"])
    kw = {k: v for k, v in cfg.items() if k not in ("h", "hm")}
    d = radiat(cfg["h"], cfg["hm"], fnot, **kw)
    o = R.radiat(cfg["h"], cfg["hm"], fnot, **kw)
    assert _close(d.atm_tmbar, o.atm_tmbar) and _close(d.ocn_tmbar, o.ocn_tmbar)
    aup = np.array([[d.aup[k][l] for l in range(nl)] for k in range(nl + 1)])
    adown = np.array([[d.adown[k - 1][l] for l in range(nl)] for k in range(1, nl + 1)])
    assert _close(aup, o.aup)
    assert _close(adown, o.adown[1:])
    assert _close([d.dup[k] for k in range(nl + 1)], o.dup)
    assert _close([d.rbetat[k] for k in range(nl - 1)], o.rbetat)
    assert _close(d.rbtmat, o.rbtmat) and _close(d.rbtmoc, o.rbtmoc)
    c = d.c
    assert c.fspco == np.copysign(cfg["fspamp"], fnot) and c.xlamda == cfg["xlamda"]
    for name, ref in (("d0up", o.d0up), ("dmdown", o.dmdown), ("dup0", o.dup[0]), ("aup00", o.aup[0, 0]),
                      ("adown10", o.adown[1, 0]), ("adown11", o.adown[1, 1])):
        assert _close(getattr(c, name), ref), name
    af, bf, df = entrain_coeff(nl, 1.0e3, cfg["tabsat"][0] - cfg["tabsat"][1], d)
    ra, rb, rd = R.entrain_coeff(nl, 1.0e3, cfg["tabsat"][0] - cfg["tabsat"][1], o)
    assert _close(af, ra) and _close(bf, rb) and _close(df, rd)


def test_mean_state_balances():
    """The mean state closes the column: the upgoing flux at the top equals
    -fsbar, and at the ocean surface the sensible + latent and radiative
    fluxes balance -fsbar too (radsubs.F90:244-336)."""
    cfg = DG
    o = R.radiat(cfg["h"], cfg["hm"], 1e-4, **{k: v for k, v in cfg.items() if k not in ("h", "hm")})
    nl = len(cfg["h"])
    assert abs(o.fupbar[nl] + cfg["fsbar"]) <= 1e-11 * abs(cfg["fsbar"])
    surf = (cfg["xlamda"] * (o.ocn_tmbar - o.atm_tmbar) + R.STEFAN * o.ocn_tmbar ** 4
            - R.bflux(o.atm_tmbar, 0.0, 0.0))
    assert abs(surf + cfg["fsbar"]) <= 1e-11 * abs(cfg["fsbar"])
    assert np.max(np.abs(o.rbalar @ np.append(o.rbetat, o.rbtmat) + 1.0)) <= 1e-12


def test_isothermal_layers_integrate_exactly():
    """gamma = 0: each layer's mean radiation is sigma/2 T^4 (1 - tau_k),
    the integral of the transmissivity, to the trapezoidal rule's error."""
    cfg = dict(DG, gamma=0.0)
    o = R.radiat(cfg["h"], cfg["hm"], 1e-4, **{k: v for k, v in cfg.items() if k not in ("h", "hm")})
    for k in range(1, 4):
        exact = R.SIGOV2 * cfg["tabsat"][k - 1] ** 4 * (1.0 - o.tauk[k])
        assert abs(o.uprad[k] - exact) <= 1e-8 * exact
        assert abs(o.dnrad[k] - exact) <= 1e-8 * exact


def test_zonal_temp_matches_oracle_and_is_odd():
    ya0, yla = 0.0, 96 * 80e3
    d = zonal_temp(96, 0.0, 80e3, 1e-4, ya0, yla, 12.0)
    o = R.zonal_temp(96, 0.0, 80e3, 1e-4, ya0, yla, 12.0)
    assert _close(d, o)
    assert np.max(np.abs(d + d[::-1])) <= 1e-13 * 12.0      # odd about the channel's middle
    assert d[0] > 0.0 > d[-1]                               # warm south in the northern hemisphere
    # an ocean centred in the channel: its wall temperatures (omlsubs.F90:38-41)
    wall = zonal_temp(512, 16 * 80e3, 10e3, 1e-4, ya0, yla, 12.0)
    assert _close(wall, R.zonal_temp(512, 16 * 80e3, 10e3, 1e-4, ya0, yla, 12.0))


def test_rejected_inputs():
    kw = {k: v for k, v in DG.items() if k not in ("h", "hm")}
    with pytest.raises(OqgError):
        radiat(DG["h"], DG["hm"], 1e-4, **dict(kw, fspamp=-1.0))      # load_rad stops on fspamp < 0
    with pytest.raises(OqgError):
        radiat(DG["h"], 2500.0, 1e-4, **kw)                          # mixed layer deeper than layer 1
    with pytest.raises(OqgError):
        radiat(DG["h"], DG["hm"], 1e-4, **dict(kw, zopt=[0.0, 3e4, 3e4, 4e4]))


def test_rbal_states():
    """The radiative-balance initial states (openqg.F90:249-306) from the
    coupled start-up: the atmosphere's layer pressures follow fsprim with
    the layer factors, layer 1 at rest; the mixed layers carry the zonal
    temperature profiles, the ocean's ends its wall temperatures."""
    from openqg_b200.params import atmos_channel, ocean_double_gyre
    from openqg_b200.radiation import coupled_start, rbal_states
    ba, bo = atmos_channel(49, 25, dx=80e3), ocean_double_gyre(129, dx=10e3)
    kw = dict(hm_a=1000.0, fsbar=-210.0, fspamp=80.0, zopt=[200.0, 3.0e4, 3.0e4, 4.0e4], gamma=1.0e-2, xlamda=35.0,
              tabsat=[330.0, 340.0, 350.0], rho_a=1.0, cp_a=1.0e3, t1_abs_o=278.0, t2_abs_o=268.0, rho_o=1.0e3,
              cp_o=4.0e3)
    rad, atm, ocn = coupled_start(ba, bo, **kw)
    p, sst, ast = rbal_states(ba, bo, rad, atm)
    o = R.radiat(ba.h, 1000.0, ba.fnot, fsbar=-210.0, fspamp=80.0, zopt=kw["zopt"], gamma=1e-2, xlamda=35.0,
                 tabsat=kw["tabsat"])
    yla = (ba.nyp - 1) * ba.dy
    fsp = 80.0 * 0.5 * np.sin(np.pi * (-0.5 * yla + np.arange(ba.nyp) * ba.dy) / yla)
    assert np.all(p[0] == 0.0)
    plf = [0.0, -ba.gp[0] * o.rbetat[0], -ba.gp[0] * o.rbetat[0] - ba.gp[1] * o.rbetat[1]]
    for k in range(3):
        assert _close(p[k], plf[k] * fsp[:, None] * np.ones((1, ba.nxp)))
    assert sst[0, 0] == ocn["sval"] and sst[-1, 0] == ocn["nval"]
    assert np.all(sst == sst[:, :1])
    assert np.array_equal(ast, atm["xc1ast"])


def test_coupled_start_keywords_fit_the_mixed_layers():
    """coupled_start's keyword dictionaries are arguments the mixed-layer
    classes take (checked by signature; no device)."""
    import inspect
    from openqg_b200.core import AtmosMixedLayer, OceanMixedLayer
    from openqg_b200.params import atmos_channel, ocean_double_gyre
    from openqg_b200.radiation import coupled_start
    ba, bo = atmos_channel(49, 25, dx=80e3), ocean_double_gyre(129, dx=10e3)
    _, atm, ocn = coupled_start(ba, bo, hm_a=1000.0, fsbar=-210.0, fspamp=80.0, zopt=[200.0, 3.0e4, 3.0e4, 4.0e4],
                                gamma=1.0e-2, xlamda=35.0, tabsat=[330.0, 340.0, 350.0], rho_a=1.0, cp_a=1.0e3,
                                t1_abs_o=278.0, t2_abs_o=268.0, rho_o=1.0e3, cp_o=4.0e3)
    for cls, kw in ((AtmosMixedLayer, atm), (OceanMixedLayer, ocn)):
        params = inspect.signature(cls.__init__).parameters
        assert set(kw) <= set(params), (cls.__name__, set(kw) - set(params))
    assert atm["xc1ast"].shape == (ba.nyp - 1, ba.nxp - 1)
    assert len(atm["aface"]) == ba.nl - 1
