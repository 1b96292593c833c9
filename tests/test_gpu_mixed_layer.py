"""The ocean mixed layer and Ekman fields on the device (oqg_ocean_forcing)
against the CPU restatement (oracle/mixed_layer.py).

Tolerances (relative L2):
  * sst, its lagged value, wekp and ent after each coupling step: 1e-12
    (FP64 arithmetic on the same inputs; sums differ in order only);
  * a coupled run (forcing then step_qg, five times) against the oracle's
    mixed layer feeding the C++ oracle's QG step: p and q 1e-11, sst 1e-11;
  * an OQG_MIXED handle (FP32 forcing fields): wekp and ent 1e-6.
"""
import numpy as np
import pytest

import oracle
from oracle.mixed_layer import OmlOracle, OmlParams, ekman
from openqg_b200.core import QG, OceanMixedLayer, OqgError, get_forcing
from openqg_b200.params import OQG_MIXED, atmos_channel, double_gyre_tau, initial_psi, ocean_double_gyre
from tests.qg_numpy import rel_l2

pytestmark = pytest.mark.gpu

TDT = 3600.0


@pytest.fixture(autouse=True)
def _need_gpu(gpu_required):
    pass


def _setup(n=65, precision=0, fluxs=True, seed=2, south=False, nl=3):
    b = ocean_double_gyre(n, dx=20.0e3, precision=precision)
    if south:                      # southern hemisphere: the northern wall may carry the flux
        b.fnot = -b.fnot
    if nl == 2:
        b.h, b.gp, b.ah2, b.ah4 = [1000.0, 3000.0], [0.02], [0.0, 0.0], [2.0e10] * 2
    elif nl == 4:
        b.h, b.gp = [300.0, 500.0, 800.0, 2400.0], [0.04, 0.02, 0.01]
        b.ah2, b.ah4 = [0.0] * 4, [2.0e10] * 4
    prm = OmlParams(hm=100.0, rho_cp=4.0e6, t1_rel=10.0, dt_12=5.0, st2d=2.0e3, st4d=1.0e11, ycexp=1.0,
                    fluxs=fluxs and not south, fluxn=south, sval=14.0, nval=8.0)
    rng = np.random.default_rng(seed)
    nyt, nxt = b.nyp - 1, b.nxp - 1
    yy = np.linspace(0.0, 1.0, nyt)[:, None]
    sst = prm.t1_rel + 2.0 + 3.0 * np.cos(np.pi * yy) + 0.3 * rng.standard_normal((nyt, nxt))
    sstm = sst + 0.05 * rng.standard_normal((nyt, nxt))
    taux, tauy = double_gyre_tau(b)
    tauy = tauy + 0.02 * rng.standard_normal(tauy.shape)
    fnet = 40.0 * rng.standard_normal((nyt, nxt))
    p = b.fnot * initial_psi(b, seed=seed)
    g = QG(b)
    g.set_state(p, p)
    m = OceanMixedLayer(g, prm.hm, prm.rho_cp, prm.t1_rel, prm.dt_12, prm.st2d, prm.st4d, prm.ycexp,
                        prm.fluxn, prm.fluxs, prm.nval, prm.sval)
    m.set_sst(sst, sstm)
    o = OmlOracle(b, prm)
    o.data, o.datam = sst.copy(), sstm.copy()
    return b, prm, g, m, o, taux, tauy, fnet, p


@pytest.mark.parametrize("south,nl", [(False, 3), (True, 3), (False, 2), (False, 4)])
def test_forcing_matches_oracle(south, nl):
    """Northern hemisphere with the southern flux condition, southern
    hemisphere with the northern one; 2, 3 and 4 layers."""
    b, prm, g, m, o, taux, tauy, fnet, _ = _setup(south=south, nl=nl)
    uek, vek, wekt, wekp = ekman(taux, tauy, b.dx, b.dy, b.fnot, prm.hm)
    ent = np.zeros((b.nl - 1,) + b.shape2)
    for it, ce in enumerate((True, False, True)):
        p1 = g.get_state()[0][0]
        m.forcing(taux, tauy, fnet, ce, TDT)
        o.step(p1, uek, vek, wekt, fnet, ce, TDT, ent)
        sst, sstm = m.get_sst()
        assert rel_l2(sst, o.data) <= 1e-12, it
        assert rel_l2(sstm, o.datam) <= 1e-12, it
        w, e = get_forcing(g)
        assert rel_l2(w, wekp) <= 1e-12
        assert rel_l2(e, ent) <= 1e-12, it
        g.step(TDT, 1)
    m.close()
    g.close()


def test_coupled_run_matches_oracle():
    """Five ocean steps of the coupled pattern: the mixed layer's forcing,
    then step_qg with it, on the device and on the CPU."""
    b, prm, g, m, o, taux, tauy, fnet, p = _setup(seed=5)
    q = oracle.Oracle(b)
    q.set_state(p, p)
    uek, vek, wekt, wekp = ekman(taux, tauy, b.dx, b.dy, b.fnot, prm.hm)
    ent = np.zeros((b.nl - 1,) + b.shape2)
    for _ in range(5):
        p1 = q.get_state()[0][0]
        o.step(p1, uek, vek, wekt, fnet, True, TDT, ent)
        q.set_forcing(wekp, ent, 0.0, 0.0)
        q.step(TDT, 1)
        m.forcing(taux, tauy, fnet, True, TDT)
        g.step(TDT, 1)
    for a, r in zip(g.get_state(), q.get_state()):
        assert rel_l2(a, r) <= 1e-11
    assert rel_l2(m.get_sst()[0], o.data) <= 1e-11
    m.close()
    g.close()


def test_mixed_precision_handle_forcing():
    b, prm, g, m, o, taux, tauy, fnet, _ = _setup(precision=OQG_MIXED, seed=7)
    uek, vek, wekt, wekp = ekman(taux, tauy, b.dx, b.dy, b.fnot, prm.hm)
    ent = np.zeros((b.nl - 1,) + b.shape2)
    p1 = g.get_state()[0][0]          # the FP32 state, widened
    m.forcing(taux, tauy, fnet, True, TDT)
    o.step(p1, uek, vek, wekt, fnet, True, TDT, ent)
    assert rel_l2(m.get_sst()[0], o.data) <= 1e-12
    w, e = get_forcing(g)
    assert rel_l2(w, wekp) <= 1e-6
    assert rel_l2(e, ent) <= 1e-6
    m.close()
    g.close()


def test_rejected_setups():
    b = ocean_double_gyre(33)
    g = QG(b)
    with pytest.raises(OqgError):        # northern flux condition in the northern hemisphere
        OceanMixedLayer(g, 100.0, 4.0e6, 10.0, 5.0, fluxn=True)
    g.close()
    c = QG(atmos_channel(33, 17))
    with pytest.raises(OqgError):        # the ocean mixed layer needs a closed box
        OceanMixedLayer(c, 100.0, 4.0e6, 10.0, 5.0)
    c.close()


# ---------------------------------------------------------------- atmosphere
from oracle.mixed_layer import AmlOracle, AmlParams, atmos_stress, ekman_cyclic, ocean_stress  # noqa: E402
from oracle.mixed_layer import RadCoeffs, compute_forcing  # noqa: E402
from openqg_b200.core import AtmosMixedLayer, xforc  # noqa: E402
from openqg_b200.params import OqgRadCoeffs  # noqa: E402

TDTA = 360.0


def _atmos_setup(seed=4, nl=3):
    b = atmos_channel(65, 33)
    if nl == 2:
        b.h, b.gp, b.ah4 = [4000.0, 5000.0], [0.8], [2.0e13] * 2
    rng = np.random.default_rng(seed)
    nyt, nxt = b.nyp - 1, b.nxp - 1
    prm = AmlParams(aface=tuple(rng.uniform(-1e-6, 1e-6, b.nl - 1)), bface=3e-7, dface=1e-5)
    xc1ast = 0.5 * rng.standard_normal((nyt, nxt))
    dtop = 50.0 * rng.standard_normal(b.shape2)
    dtop[:, -1] = dtop[:, 0]
    y = np.arange(b.nyp) * b.dy
    taux = np.repeat((0.1 * np.sin(np.pi * y / y[-1]))[:, None], b.nxp, axis=1) + 0.01 * rng.standard_normal(b.shape2)
    tauy = 0.01 * rng.standard_normal(b.shape2)
    taux[:, -1] = taux[:, 0]
    tauy[:, -1] = tauy[:, 0]
    fnet = 30.0 * rng.standard_normal((nyt, nxt))
    ast = prm.t1_rel - 2.0 + rng.standard_normal((nyt, nxt))
    astm = ast + 0.1 * rng.standard_normal((nyt, nxt))
    hmx = prm.hm + 50.0 * rng.standard_normal((nyt, nxt))
    hmxm = hmx + 5.0 * rng.standard_normal((nyt, nxt))
    p = b.fnot * 30.0 * initial_psi(b, seed=seed)
    g = QG(b)
    g.set_state(p, p)
    m = AtmosMixedLayer(g, xc1ast, dtop, hm=prm.hm, rho_cp=prm.rho_cp, t1_rel=prm.t1_rel, dt_12=prm.dt_12,
                        hmamin=prm.hmamin, hmadmp=prm.hmadmp, xcexp=prm.xcexp, at2d=prm.at2d, at4d=prm.at4d,
                        ahmd=prm.ahmd, aface=prm.aface, bface=prm.bface, dface=prm.dface)
    m.set_state(ast, astm, hmx, hmxm)
    o = AmlOracle(b, prm, xc1ast, dtop)
    o.ast, o.astm, o.hmx, o.hmxm = ast.copy(), astm.copy(), hmx.copy(), hmxm.copy()
    return b, prm, g, m, o, taux, tauy, fnet, p


def _eta(b, pm):
    return np.stack([(pm[k] - pm[k + 1]) / b.gp[k] for k in range(b.nl - 1)])


@pytest.mark.parametrize("nl", [3, 2])
def test_atmos_forcing_matches_oracle(nl):
    b, prm, g, m, o, taux, tauy, fnet, _ = _atmos_setup(nl=nl)
    uek, vek, wekt, wekp, txis, txin = ekman_cyclic(taux, tauy, b.dx, b.dy, b.fnot, prm.hm)
    ent = np.zeros((b.nl - 1,) + b.shape2)
    for it, ce in enumerate((True, False, True)):
        p, pm, _, _ = g.get_state()
        m.forcing(taux, tauy, fnet, ce, TDTA)
        o.step(p[0], uek, vek, wekt, _eta(b, pm), fnet, ce, TDTA, ent)
        for name, a, r in zip(("ast", "astm", "hmixa", "hmixam"), m.get_state(), (o.ast, o.astm, o.hmx, o.hmxm)):
            assert rel_l2(a, r) <= 1e-12, (it, name)
        w, e = get_forcing(g)
        assert rel_l2(w, wekp) <= 1e-12
        assert rel_l2(e, ent) <= 1e-12, it
        g.step(TDTA, 1)
    m.close()
    g.close()


def test_atmos_coupled_run_matches_oracle():
    """Four atmosphere steps of the coupled pattern: the mixed layer's forcing
    (with txis, txin), then step_qg, on the device and on the CPU."""
    b, prm, g, m, o, taux, tauy, fnet, p = _atmos_setup(seed=6)
    q = oracle.Oracle(b)
    q.set_state(p, p)
    uek, vek, wekt, wekp, txis, txin = ekman_cyclic(taux, tauy, b.dx, b.dy, b.fnot, prm.hm)
    ent = np.zeros((b.nl - 1,) + b.shape2)
    for _ in range(4):
        qp, qpm, _, _ = q.get_state()
        o.step(qp[0], uek, vek, wekt, _eta(b, qpm), fnet, True, TDTA, ent)
        q.set_forcing(wekp, ent, txis, txin)
        q.step(TDTA, 1)
        m.forcing(taux, tauy, fnet, True, TDTA)
        g.step(TDTA, 1)
    for a, r in zip(g.get_state(), q.get_state()):
        assert rel_l2(a, r) <= 1e-11
    assert rel_l2(m.get_state()[0], o.ast) <= 1e-11
    m.close()
    g.close()


def test_atmos_rejects_a_box():
    g = QG(ocean_double_gyre(33))
    with pytest.raises(OqgError):
        AtmosMixedLayer(g, np.zeros((32, 32)), None, hm=1000.0, rho_cp=1e3, t1_rel=-5.0, dt_12=20.0, hmamin=100.0,
                        hmadmp=0.5, xcexp=1.0, at2d=0.0, at4d=0.0, ahmd=0.0, aface=(0.0, 0.0), bface=0.0, dface=0.0)
    g.close()


def test_atmos_forcing_with_its_own_stress():
    """taux = tauy = None: the stress that xforc computed on the device
    from the atmosphere's lagged layer-1 pressure by the drag law."""
    b, prm, g, m, o, _, _, fnet, _ = _atmos_setup(seed=8)
    ent = np.zeros((b.nl - 1,) + b.shape2)
    g.step(TDTA, 2)                          # a lagged pressure unlike the current one
    for ce in (True, True):
        p, pm, _, _ = g.get_state()
        taux, tauy = atmos_stress(pm[0], b, 1.3e-3, prm.hm)
        uek, vek, wekt, wekp, _, _ = ekman_cyclic(taux, tauy, b.dx, b.dy, b.fnot, prm.hm)
        xforc(m)
        m.forcing(None, None, fnet, ce, TDTA)
        o.step(p[0], uek, vek, wekt, _eta(b, pm), fnet, ce, TDTA, ent)
        assert rel_l2(m.get_state()[0], o.ast) <= 1e-12
        w, e = get_forcing(g)
        assert rel_l2(w, wekp) <= 1e-12
        assert rel_l2(e, ent) <= 1e-12
        g.step(TDTA, 1)
    m.close()
    g.close()


def test_ocean_stress_from_the_coupled_atmosphere():
    """The ocean (129x129 at 10 km) coupled to an atmosphere channel (49x25 at
    80 km): the ocean's stress from xforc, computed on the device from the
    atmosphere's lagged layer-1 pressure through the bicubic interpolation
    and the drag law."""
    ba = atmos_channel(49, 25, dx=80e3)
    ga = QG(ba)
    pa = ba.fnot * 30.0 * initial_psi(ba, seed=3)
    ga.set_state(pa, pa)
    y = np.arange(ba.nyp) * ba.dy
    txa = np.repeat((0.05 * np.sin(np.pi * y / y[-1]))[:, None], ba.nxp, axis=1)
    w, ts, tn = oracle.ekman_from_tau(ba, txa, np.zeros_like(txa))
    ga.set_forcing(w, None, ts, tn)
    ga.step(TDTA, 3)                           # p and pm differ
    aprm = AmlParams(aface=(1e-7, -1e-7), bface=1e-7, dface=1e-6)
    aml = AtmosMixedLayer(ga, np.zeros((ba.nyp - 1, ba.nxp - 1)), None, hm=aprm.hm, rho_cp=aprm.rho_cp,
                          t1_rel=aprm.t1_rel, dt_12=aprm.dt_12, hmamin=aprm.hmamin, hmadmp=aprm.hmadmp,
                          xcexp=aprm.xcexp, at2d=aprm.at2d, at4d=aprm.at4d, ahmd=aprm.ahmd, aface=aprm.aface,
                          bface=aprm.bface, dface=aprm.dface, cdat=1.3e-3)
    prm = OmlParams(hm=100.0, rho_cp=4.0e6, t1_rel=10.0, dt_12=5.0, st2d=2.0e3, st4d=1.0e11, ycexp=1.0)
    b = ocean_double_gyre(129, dx=10.0e3)
    g = QG(b)
    p = b.fnot * initial_psi(b, seed=9)
    g.set_state(p, p)
    m = OceanMixedLayer(g, prm.hm, prm.rho_cp, prm.t1_rel, prm.dt_12, prm.st2d, prm.st4d, prm.ycexp,
                        prm.fluxn, prm.fluxs, prm.nval, prm.sval)
    sst = prm.t1_rel + 2.0 + np.zeros((b.nyp - 1, b.nxp - 1))
    m.set_sst(sst, sst)
    o = OmlOracle(b, prm)
    o.data, o.datam = sst.copy(), sst.copy()
    fnet = np.zeros((b.nyp - 1, b.nxp - 1))
    m.couple(aml, 1.2e-3)
    ent = np.zeros((b.nl - 1,) + b.shape2)
    for _ in range(2):
        pma = ga.get_state()[1][0]
        taux, tauy = ocean_stress(pma, ba, b, 1.3e-3, aprm.hm, 1.2e-3)
        uek, vek, wekt, wekp = ekman(taux, tauy, b.dx, b.dy, b.fnot, prm.hm)
        p1 = g.get_state()[0][0]
        xforc(aml, m)
        m.forcing(None, None, fnet, True, TDT)
        o.step(p1, uek, vek, wekt, fnet, True, TDT, ent)
        w, e = get_forcing(g)
        assert rel_l2(w, wekp) <= 1e-12
        assert rel_l2(e, ent) <= 1e-12
        assert rel_l2(m.get_sst()[0], o.data) <= 1e-12
        g.step(TDT, 1)
        aml.forcing(None, None, np.zeros((ba.nyp - 1, ba.nxp - 1)), True, TDTA)
        ga.step(TDTA, 1)
    for x in (m, aml, g, ga):
        x.close()


RAD = RadCoeffs(fspco=80.0, xlamda=35.0, d0up=5.5, dmdown=3.5, dup0=2.5, aup00=-0.03, adown10=0.02, adown11=0.01)


def _rad_c():
    return OqgRadCoeffs(*[getattr(RAD, f) for f, _ in OqgRadCoeffs._fields_])


def _coupled_pair(seed, topography=True, precision=0):
    """An ocean box (129x129 at 10 km) under an atmosphere channel (49x25 at
    80 km), both mixed layers coupled, lagged states unlike the current
    ones; the channel's QG state stepped three times on the device and by
    the C++ oracle alike."""
    rng = np.random.default_rng(seed)
    ba = atmos_channel(49, 25, dx=80e3, precision=precision)
    ga, qa = QG(ba), oracle.Oracle(ba)
    pa = ba.fnot * 30.0 * initial_psi(ba, seed=seed)
    ga.set_state(pa, pa)
    qa.set_state(pa, pa)
    y = np.arange(ba.nyp) * ba.dy
    txa = np.repeat((0.05 * np.sin(np.pi * y / y[-1]))[:, None], ba.nxp, axis=1)
    w, ts, tn = oracle.ekman_from_tau(ba, txa, np.zeros_like(txa))
    ga.set_forcing(w, None, ts, tn)
    qa.set_forcing(w, np.zeros((ba.nl - 1,) + ba.shape2), ts, tn)
    ga.step(TDTA, 3)
    qa.step(TDTA, 3)
    aprm = AmlParams(aface=(1e-7, -1e-7), bface=1e-7, dface=1e-6)
    nyta, nxta = ba.nyp - 1, ba.nxp - 1
    dtop = None
    if topography:
        dtop = 50.0 * rng.standard_normal(ba.shape2)
        dtop[:, -1] = dtop[:, 0]
    aml = AtmosMixedLayer(ga, np.zeros((nyta, nxta)), dtop, hm=aprm.hm, rho_cp=aprm.rho_cp, t1_rel=aprm.t1_rel,
                          dt_12=aprm.dt_12, hmamin=aprm.hmamin, hmadmp=aprm.hmadmp, xcexp=aprm.xcexp,
                          at2d=aprm.at2d, at4d=aprm.at4d, ahmd=aprm.ahmd, aface=aprm.aface, bface=aprm.bface,
                          dface=aprm.dface, cdat=1.3e-3)
    ya = np.linspace(0.0, 1.0, nyta)[:, None]
    ast = -8.0 + 2.0 * np.cos(np.pi * ya) + 0.3 * rng.standard_normal((nyta, nxta))
    astm = ast + 0.05 * rng.standard_normal((nyta, nxta))
    hmx = aprm.hm + 50.0 * rng.standard_normal((nyta, nxta))
    hmxm = hmx + 5.0 * rng.standard_normal((nyta, nxta))
    aml.set_state(ast, astm, hmx, hmxm)
    oa = AmlOracle(ba, aprm, np.zeros((nyta, nxta)), dtop if dtop is not None else np.zeros(ba.shape2))
    oa.ast, oa.astm, oa.hmx, oa.hmxm = ast.copy(), astm.copy(), hmx.copy(), hmxm.copy()
    prm = OmlParams(hm=100.0, rho_cp=4.0e6, t1_rel=10.0, dt_12=5.0, st2d=2.0e3, st4d=1.0e11, ycexp=1.0)
    b = ocean_double_gyre(129, dx=10.0e3, precision=precision)
    g, qo = QG(b), oracle.Oracle(b)
    p = b.fnot * initial_psi(b, seed=seed + 1)
    g.set_state(p, p)
    qo.set_state(p, p)
    m = OceanMixedLayer(g, prm.hm, prm.rho_cp, prm.t1_rel, prm.dt_12, prm.st2d, prm.st4d, prm.ycexp,
                        prm.fluxn, prm.fluxs, prm.nval, prm.sval)
    nyt, nxt = b.nyp - 1, b.nxp - 1
    yo = np.linspace(0.0, 1.0, nyt)[:, None]
    sst = 12.0 + 3.0 * np.cos(np.pi * yo) + 0.3 * rng.standard_normal((nyt, nxt))
    sstm = sst + 0.05 * rng.standard_normal((nyt, nxt))
    m.set_sst(sst, sstm)
    oo = OmlOracle(b, prm)
    oo.data, oo.datam = sst.copy(), sstm.copy()
    m.couple(aml, 1.2e-3)
    return dict(ba=ba, ga=ga, qa=qa, aml=aml, oa=oa, aprm=aprm, dtop=dtop,
                b=b, g=g, qo=qo, m=m, oo=oo, prm=prm)


@pytest.mark.parametrize("topography,source", [(True, "fixed"), (False, "fixed"), (True, "radiat")])
def test_coupled_fluxes_match_oracle(topography, source):
    """compute_forcing on the device: both mixed layers' net heat fluxes
    against the restatement, before and after the atmosphere steps; the
    radiation coefficients fixed, or from the radiative start-up with the
    reference's atmosphere parameters (data/basin/atm_dg.cdl)."""
    c = _coupled_pair(seed=11, topography=topography)
    ba, b, m, aml, ga = c["ba"], c["b"], c["m"], c["aml"], c["ga"]
    rc, rad = _rad_c(), RAD
    if source == "radiat":
        from openqg_b200.radiation import radiat
        rc = radiat(ba.h, 1000.0, ba.fnot, fsbar=-210.0, fspamp=80.0, zopt=[200.0, 3.0e4, 3.0e4, 4.0e4],
                    gamma=1.0e-2, xlamda=35.0, tabsat=[330.0, 340.0, 350.0]).c
        rad = RadCoeffs(*[getattr(rc, f) for f, _ in OqgRadCoeffs._fields_])
    for it in range(2):
        m.compute_forcing(rc)
        fo, fa = m.get_fluxes()
        _, astm, _, hmxm = aml.get_state()
        sstm = m.get_sst()[1]
        pma = ga.get_state()[1]
        ro, ra = compute_forcing(sstm, astm, hmxm, pma, ba, b, rad, c["aprm"].hm, c["aprm"].hmadmp, c["dtop"])
        assert rel_l2(fo, ro) <= 1e-12, it
        assert rel_l2(fa, ra) <= 1e-12, it
        xforc(aml, m)
        aml.forcing(None, None, None, True, TDTA)
        ga.step(TDTA, 1)
    for k in ("m", "aml", "g", "ga"):
        c[k].close()


@pytest.mark.parametrize("precision,tol,nocean", [(0, 1e-11, 3), (OQG_MIXED, 1e-5, 3), (OQG_MIXED, 1e-5, 10)],
                         ids=["fp64_3", "mixed_3", "mixed_10"])
def test_coupled_exchange_matches_oracle(precision, tol, nocean):
    """Ocean steps of the coupled driver (driver.F90:33-143) with two
    atmosphere steps each, every exchange on the device: xforc (both
    stresses), compute_forcing (both fluxes), the mixed layers and QG steps
    of both basins; against the restatements and the C++ oracle's FP64 QG
    steps.  FP64 handles within 1e-11 after 3 ocean steps; FP32 state
    storage (OQG_MIXED, the coupled configuration's FP32-bulk form) within
    1e-5 after 3 and after the configuration's 10 coupled ocean steps."""
    c = _coupled_pair(seed=13, precision=precision)
    ba, b, aprm, prm = c["ba"], c["b"], c["aprm"], c["prm"]
    ga, qa, aml, oa, g, qo, m, oo = (c[k] for k in ("ga", "qa", "aml", "oa", "g", "qo", "m", "oo"))
    enta = np.zeros((ba.nl - 1,) + ba.shape2)
    ento = np.zeros((b.nl - 1,) + b.shape2)
    nstr = 2
    for _ in range(nocean):
        # the oracle's ocean step
        pma = qa.get_state()[1]
        tax, tay = atmos_stress(pma[0], ba, 1.3e-3, aprm.hm)
        tox, toy = ocean_stress(pma[0], ba, b, 1.3e-3, aprm.hm, 1.2e-3)
        fo, fa = compute_forcing(oo.datam, oa.astm, oa.hmxm, pma, ba, b, RAD, aprm.hm, aprm.hmadmp, c["dtop"])
        ua, va, wta, wpa, tsa, tna = ekman_cyclic(tax, tay, ba.dx, ba.dy, ba.fnot, aprm.hm)
        uo, vo, wto, wpo = ekman(tox, toy, b.dx, b.dy, b.fnot, prm.hm)
        for s in range(nstr):
            p, pm = qa.get_state()[:2]
            oa.step(p[0], ua, va, wta, _eta(ba, pm), fa, True, TDTA, enta)
            qa.set_forcing(wpa, enta, tsa, tna)
            qa.step(TDTA, 1)
            if s == 0:
                oo.step(qo.get_state()[0][0], uo, vo, wto, fo, True, TDT, ento)
                qo.set_forcing(wpo, ento, 0.0, 0.0)
                qo.step(TDT, 1)
        # the same on the device
        xforc(aml, m)
        m.compute_forcing(_rad_c())
        for s in range(nstr):
            aml.forcing(None, None, None, True, TDTA)
            ga.step(TDTA, 1)
            if s == 0:
                m.forcing(None, None, None, True, TDT)
                g.step(TDT, 1)
    for a, r in zip(ga.get_state(), qa.get_state()):
        assert rel_l2(a, r) <= tol
    for a, r in zip(g.get_state(), qo.get_state()):
        assert rel_l2(a, r) <= tol
    assert rel_l2(m.get_sst()[0], oo.data) <= tol
    assert rel_l2(aml.get_state()[0], oa.ast) <= tol
    assert rel_l2(aml.get_state()[2], oa.hmx) <= tol
    for k in ("m", "aml", "g", "ga"):
        c[k].close()


def test_compute_forcing_needs_a_coupled_atmosphere():
    g = QG(ocean_double_gyre(33))
    m = OceanMixedLayer(g, 100.0, 4.0e6, 10.0, 5.0)
    with pytest.raises(OqgError):
        m.compute_forcing(_rad_c())
    m.close()
    g.close()


def test_tau_udiff_stresses_match_oracle():
    """tau_udiff: the stress of the atmosphere-ocean velocity difference
    (compute_udiff), for both basins, through each handle's Ekman pumping;
    the atmosphere's stress over the ocean is the ocean-resolution one."""
    c = _coupled_pair(seed=17)
    ba, b, aprm, prm = c["ba"], c["b"], c["aprm"], c["prm"]
    ga, aml, g, m = c["ga"], c["aml"], c["g"], c["m"]
    g.step(TDT, 2)                         # the ocean's lagged pressure unlike its current one
    m.tau_udiff(True)
    for _ in range(2):
        pma, pmo = ga.get_state()[1], g.get_state()[1]
        tax, tay = atmos_stress(pma[0], ba, 1.3e-3, aprm.hm)
        tox, toy = ocean_stress(pma[0], ba, b, 1.3e-3, aprm.hm, 1.2e-3, pmo1=pmo[0], hmo=prm.hm,
                                atmos_tau=(tax, tay))
        wpo = ekman(tox, toy, b.dx, b.dy, b.fnot, prm.hm)[3]
        wpa = ekman_cyclic(tax, tay, ba.dx, ba.dy, ba.fnot, aprm.hm)[3]
        xforc(aml, m)
        m.forcing(None, None, np.zeros((b.nyp - 1, b.nxp - 1)), True, TDT)
        aml.forcing(None, None, np.zeros((ba.nyp - 1, ba.nxp - 1)), True, TDTA)
        assert rel_l2(get_forcing(g)[0], wpo) <= 1e-12
        assert rel_l2(get_forcing(ga)[0], wpa) <= 1e-12
        g.step(TDT, 1)
        ga.step(TDTA, 1)
    for k in ("m", "aml", "g", "ga"):
        c[k].close()
