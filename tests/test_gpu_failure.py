"""Failure detection of the bounded device waits, without a GPU fault.

The vorticity kernel waits for its tile loads on an mbarrier with a bounded
number of polls.  oqg_set_wait_limit(h, 0) makes every first wait run out at
once: each CTA then drains the copies it has in flight (full limit), sets the
device error word and returns, so the context stays usable.  The host must
see OQG_ETIMEOUT from oqg_sync, the error word must be cleared by that
report, and after the default limit is restored and the state set again the
handle must step exactly like the oracle.
"""
import numpy as np
import pytest

import oracle
from openqg_b200.core import QG, OqgError, lib
from openqg_b200.params import double_gyre_tau, initial_psi, ocean_double_gyre
from tests.qg_numpy import rel_l2

pytestmark = pytest.mark.gpu

OQG_ETIMEOUT = 4


@pytest.fixture(autouse=True)
def _need_gpu(gpu_required):
    pass


def _inputs(b):
    p = b.fnot * initial_psi(b, 4)
    w, ts, tn = oracle.ekman_from_tau(b, *double_gyre_tau(b))
    return p, w, ts, tn


@pytest.mark.parametrize("n", [129, 513])
def test_wait_timeout_is_reported_then_cleared(n):
    b = ocean_double_gyre(n, dx=20e3 if n == 129 else 10e3)
    p, w, ts, tn = _inputs(b)
    g = QG(b)
    g.set_state(p, p)
    g.set_forcing(w, None, ts, tn)
    L = lib()
    assert L.oqg_set_wait_limit(g.h, 0) == 0
    g.step(3600.0, 1)
    assert L.oqg_sync(g.h) == OQG_ETIMEOUT
    assert b"bounded device wait" in L.oqg_last_error()
    # the report cleared the error word
    assert L.oqg_sync(g.h) == 0
    # a step through the Python mirror raises the same code
    g.step(3600.0, 1)
    with pytest.raises(OqgError) as ei:
        g.sync()
    assert ei.value.code == OQG_ETIMEOUT
    # default limit again: the handle is usable and exact after a new state
    assert L.oqg_set_wait_limit(g.h, -1) == 0
    o = oracle.Oracle(b)
    for x in (g, o):
        x.set_state(p, p)
        x.set_forcing(w, None, ts, tn)
        x.set_step_index(0)
        x.step(3600.0, 3)
    g.sync()
    for a, r in zip(g.get_state(), o.get_state()):
        assert rel_l2(a, r) <= 1e-12
    assert np.all(np.isfinite(g.get_state()[0]))
    g.close()
    o.close()
