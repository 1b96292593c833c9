"""One model year of the 129x129x3 double gyre (dt = 1800 s, 17,520 steps),
CUDA path against the FP64 oracle on the same seeded inputs.

The flow is chaotic, so the states drift apart bit by bit; the contract is on
the basin integrals: kinetic energy and meridional transport (upper-layer
stream-function range, qg_monitor.F90:331-376) within 1%, compared as means
over the last 30 days of daily samples.  The oracle part takes about a
minute and a half of one host core.
"""
import numpy as np
import pytest

import oracle
from openqg_b200.core import QG
from openqg_b200.params import double_gyre_tau, initial_psi, ocean_double_gyre

pytestmark = pytest.mark.gpu

STEPS_PER_DAY = 48          # dt = 1800 s
DAYS = 365
TAIL_DAYS = 30
TOL = 0.01


def _series(x, days):
    ke, tr = [], []
    for _ in range(days):
        x.step(3600.0, STEPS_PER_DAY)
        d = x.diag()
        ke.append(float(np.sum(d["ekei"])))
        tr.append(float(d["sfmax"][0] - d["sfmin"][0]))
    return np.array(ke), np.array(tr)


def test_one_year_ke_and_transport_within_one_percent(gpu_required):
    b = ocean_double_gyre(129)
    p = b.fnot * initial_psi(b, 1)
    w, ts, tn = oracle.ekman_from_tau(b, *double_gyre_tau(b))
    g, o = QG(b), oracle.Oracle(b)
    for x in (g, o):
        x.set_state(p, p)
        x.set_forcing(w, None, ts, tn)
    ke_g, tr_g = _series(g, DAYS)
    ke_o, tr_o = _series(o, DAYS)
    assert g.step_index() == DAYS * STEPS_PER_DAY
    assert np.all(np.isfinite(ke_g)) and g.check_finite() == 0
    mk_g, mk_o = ke_g[-TAIL_DAYS:].mean(), ke_o[-TAIL_DAYS:].mean()
    mt_g, mt_o = tr_g[-TAIL_DAYS:].mean(), tr_o[-TAIL_DAYS:].mean()
    assert abs(mk_g - mk_o) <= TOL * abs(mk_o), (mk_g, mk_o)
    assert abs(mt_g - mt_o) <= TOL * abs(mt_o), (mt_g, mt_o)
    g.close()
