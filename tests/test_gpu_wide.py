"""The eddy-resolving grid, 2049 x 2049 x 3 (dx = 5 km, ah4 = 1e9): its
inverse transforms keep the modal rows in a global buffer because they no
longer fit in shared memory.  One FP64 step and the modal solves are checked
against the oracle with the parity tolerances, and the mixed-precision
handle against the FP64 oracle at the 1e-5 bound on psi."""
import numpy as np
import pytest

import oracle
from openqg_b200.core import QG
from openqg_b200.params import OQG_MIXED, double_gyre_tau, initial_psi, ocean_double_gyre
from tests.qg_numpy import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu(gpu_required):
    pass


def _wide(precision=0):
    return ocean_double_gyre(2049, dx=5e3, ah4=1e9, precision=precision)


def test_wide_grid_step_matches_oracle():
    b = _wide()
    p = b.fnot * initial_psi(b, 2)
    w, ts, tn = oracle.ekman_from_tau(b, *double_gyre_tau(b))
    g, o = QG(b), oracle.Oracle(b)
    for x in (g, o):
        x.set_state(p, p)
        x.set_forcing(w, None, ts, tn)
    # the inverse transforms run as a launch of their own at this width
    assert g.step_launches() == 5
    g.step(1200.0, 1)
    o.step(1200.0, 1)
    for name, a, c in zip(("p", "pm", "q", "qm"), g.get_state(), o.get_state()):
        assert rel_l2(a, c) <= 1e-12, name
    g.close()


def test_wide_grid_modal_solve_matches_oracle():
    b = _wide()
    g, o = QG(b), oracle.Oracle(b)
    rhs = np.random.default_rng(3).random(b.shape2)
    for m in (1, 3):
        assert rel_l2(g.solve_inhomog_eqn(m, rhs), o.solve_inhomog(m, rhs)) <= 1e-13, m
    g.close()


def test_wide_grid_mixed_precision_matches_oracle():
    """FP32 bulk arithmetic at 2049^2: psi within 1e-5 relative L2 of the
    FP64 oracle after each of two steps (tests/test_gpu_mixed_errors.py
    states the error of every field over 10 steps)."""
    bm, b = _wide(OQG_MIXED), _wide()
    p = b.fnot * initial_psi(b, 2)
    w, ts, tn = oracle.ekman_from_tau(b, *double_gyre_tau(b))
    g, o = QG(bm), oracle.Oracle(b)
    for x in (g, o):
        x.set_state(p, p)
        x.set_forcing(w, None, ts, tn)
    for _ in range(2):
        g.step(1200.0, 1)
        o.step(1200.0, 1)
        P, _, Q, _ = g.get_state()
        Po, _, Qo, _ = o.get_state()
        assert rel_l2(P, Po) <= 1e-5
        assert rel_l2(Q, Qo) <= 1e-5
    assert g.check_finite() == 0
    g.close()
