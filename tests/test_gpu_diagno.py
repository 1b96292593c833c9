"""Device qg_diagno (oqg_diagno) against the oracle's restatement of
qg_monitor.F90:219-383: forcing means, interface displacement and its
energy rate, wind work, energetics, jet, transports, bottom drag and the
channel continuity check, on a box with entrainment and a channel."""
import numpy as np
import pytest

import oracle
from openqg_b200.core import QG
from openqg_b200.params import atmos_channel, double_gyre_tau, initial_psi, ocean_double_gyre
from tests.test_gpu_parity import _channel_tau, _ent

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu(gpu_required):
    pass


# area integrals are summed by rows on the device and by the reference's
# whole-array order in the oracle: relative agreement to rounding
RTOL = 1e-9


def _close(a, c, name, scale=None):
    a, c = np.asarray(a, dtype=float), np.asarray(c, dtype=float)
    scale = max(np.abs(c).max(), 1e-300) if scale is None else scale
    assert np.allclose(a, c, rtol=RTOL, atol=RTOL * scale), (name, a, c)


def _scales(d, state):
    """Magnitudes against which near-zero signed means are compared: the
    mean of |field| for a signed mean, the field RMS for layer averages."""
    p, _, q, _ = state
    return dict(wepm=d["wapm"], entm=d["enam"], etam=np.sqrt(np.max(d["et2m"])),
                pken=abs(d["pken"]) + 1e-300, pavg=np.sqrt(np.mean(p ** 2)), qavg=np.sqrt(np.mean(q ** 2)),
                circ=np.max(np.abs(d["sfmax"] - d["sfmin"])), ctot=np.max(np.abs(d["sfmax"] - d["sfmin"])))


@pytest.mark.parametrize("kind", ["box", "channel"])
def test_diagno_matches_oracle(kind):
    if kind == "box":
        b = ocean_double_gyre(97)
        taux, tauy = double_gyre_tau(b)
        amp, tdt = 1.0, 3600.0
    else:
        b = atmos_channel(97, 65)
        taux, tauy = _channel_tau(b)
        amp, tdt = 30.0, 360.0
    b.ah2 = [50.0, 20.0, 10.0]
    p = b.fnot * initial_psi(b, 4) * amp
    pm = 0.5 * p + 0.25 * b.fnot * initial_psi(b, 9) * amp
    w, ts, tn = oracle.ekman_from_tau(b, taux, tauy)
    e = _ent(b, 2)
    g, o = QG(b), oracle.Oracle(b)
    for x in (g, o):
        x.set_state(p, pm)
        x.set_forcing(w, e, ts, tn)
        x.step(tdt, 3)
    dg, mg = g.diagno(taux, tauy, tsec=3 * tdt, tdt=tdt)
    do, mo = o.diagno(taux, tauy, tsec=3 * tdt, tdt=tdt)
    g.step(tdt, 2)
    o.step(tdt, 2)
    dg, _ = g.diagno(taux, tauy, tsec=5 * tdt, tdt=tdt, mon=mg)   # pket from the two calls
    do, _ = o.diagno(taux, tauy, tsec=5 * tdt, tdt=tdt, mon=mo)
    sc = _scales(do, o.get_state())
    for key in dg:
        if key == "pos":
            assert np.array_equal(dg[key], do[key]), (key, dg[key], do[key])
        elif key in ("ermas", "emfr"):
            continue
        else:
            _close(dg[key], do[key], key, sc.get(key))
    if b.cyclic:
        # continuity error: a difference of two area integrals, so absolute
        scale = abs(mg.pavg[0]) * (b.nxp - 1) * (b.nyp - 1) * b.dx * b.dy
        assert np.allclose(dg["ermas"], do["ermas"], rtol=0, atol=1e-10 * scale)
    # the record agrees with the simpler diag entry point
    d = g.diag()
    _close(dg["ekei"], d["ekei"], "ekei vs diag")
    g.close()


def test_valids_extremes_and_bounds():
    """valids (valsubs.F90:46-139): the extremes equal numpy's over the state,
    a bound below an extreme flags the state, and a NaN does too."""
    b = ocean_double_gyre(65)
    p = b.fnot * initial_psi(b, 6)
    w, ts, tn = oracle.ekman_from_tau(b, *double_gyre_tau(b))
    g = QG(b)
    g.set_state(p, p)
    g.set_forcing(w, None, ts, tn)
    g.step(3600.0, 3)
    P, _, Q, _ = g.get_state()
    ok, ext, bad = g.valids(1e30, 1e30, 1e30)
    assert ok and bad == 0
    assert ext["pmin"] == P.min() and ext["pmax"] == P.max()
    assert ext["qmin"] == Q.min() and ext["qmax"] == Q.max()
    assert ext["wmin"] == w.min() and ext["wmax"] == w.max()
    ok, _, _ = g.valids(0.5 * max(abs(P.min()), abs(P.max())), 1e30, 1e30)
    assert not ok
    P2, PM2, Q2, QM2 = g.get_state()
    c = g.constraints()
    P2[1, 10, 10] = np.nan
    g.set_state_full(P2, PM2, Q2, QM2, c["dpi"], c["dpip"])
    ok, _, bad = g.valids(1e30, 1e30, 1e30)
    assert not ok and bad == 1
    g.close()
