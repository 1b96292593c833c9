"""The mixed-precision step (OQG_MIXED: FP32 state, stencils, Jacobian and
x-transforms; FP64 vertical-mode projection, tridiagonal solves and
compensated constraint and area integrals) against the FP64 oracle, field
by field, at the coupled configuration's ocean (513 x 513 x 3, dx 10 km) and
the eddy-resolving box (2049 x 2049 x 3, dx 5 km, ah4 1e9).

Two measures, each asserted and printed as a table row (run with -s):
  * run: both start from the same state and take 10 steps; the errors after
    step 1 and step 10;
  * per step: each of 3 steps starts the mixed handle from the oracle's
    state (rounded to FP32 storage) and compares one step.
psi (= p / f0) must stay within 1e-5 relative L2 in both, every step.
"""
import numpy as np
import pytest

import oracle
from openqg_b200.core import QG
from openqg_b200.params import OQG_MIXED, double_gyre_tau, initial_psi, ocean_double_gyre
from tests.qg_numpy import rel_l2

pytestmark = pytest.mark.gpu

PSI_TOL = 1e-5

CASES = [
    ("box513", dict(n=513, dx=10e3, ah4=2.0e10), 3600.0),
    ("box2049", dict(n=2049, dx=5e3, ah4=1.0e9), 1200.0),
]


@pytest.fixture(autouse=True)
def _need_gpu(gpu_required):
    pass


def _pair(kw):
    bm = ocean_double_gyre(kw["n"], dx=kw["dx"], ah4=kw["ah4"], precision=OQG_MIXED)
    b64 = ocean_double_gyre(kw["n"], dx=kw["dx"], ah4=kw["ah4"])
    p = b64.fnot * initial_psi(b64, 2)
    w, ts, tn = oracle.ekman_from_tau(b64, *double_gyre_tau(b64))
    g, o = QG(bm), oracle.Oracle(b64)
    for x in (g, o):
        x.set_state(p, p)
        x.set_forcing(w, None, ts, tn)
    return g, o


def _rel_max(a, r):
    a, r = np.asarray(a, float), np.asarray(r, float)
    return float(np.abs(a - r).max() / max(np.abs(r).max(), 1e-300))


def field_errors(g, o):
    """Relative errors of the mixed handle against the oracle: L2 over the
    field for p, pm, q, qm; max-norm over layers for the mass-constraint
    scalars and qg's kinetic energy and stream-function extrema."""
    out = {name: rel_l2(a, r) for name, a, r in zip(("p", "pm", "q", "qm"), g.get_state(), o.get_state())}
    cg, co = g.constraints(), o.get_constraints()
    out["dpi"] = _rel_max(cg["dpi"], co["dpi"])
    dg, do = g.diag(), o.diag()
    for key in ("ekei", "sfmin", "sfmax"):
        out[key] = _rel_max(dg[key], do[key])
    return out


FIELDS = ("p", "pm", "q", "qm", "dpi", "ekei", "sfmin", "sfmax")


def _row(case, what, e):
    return "| %s | %s | " % (case, what) + " | ".join("%.1e" % e[k] for k in FIELDS) + " |"


@pytest.mark.parametrize("case,kw,tdt", CASES, ids=[c[0] for c in CASES])
def test_mixed_run_errors_per_field(case, kw, tdt):
    g, o = _pair(kw)
    rows = []
    for s in range(1, 11):
        g.step(tdt, 1)
        o.step(tdt, 1)
        e = field_errors(g, o)
        assert e["p"] <= PSI_TOL, "step %d: psi rel L2 %.2e" % (s, e["p"])
        if s in (1, 10):
            rows.append(_row(case, "run, step %d" % s, e))
    print("\n" + "\n".join(rows))
    g.close()
    o.close()


@pytest.mark.parametrize("case,kw,tdt", CASES, ids=[c[0] for c in CASES])
def test_mixed_single_step_errors_per_field(case, kw, tdt):
    g, o = _pair(kw)
    worst = {}
    for s in range(3):
        p, pm, q, qm = o.get_state()
        c = o.get_constraints()
        g.set_state_full(p, pm, q, qm, c["dpi"], c["dpip"])
        g.set_step_index(s)
        o.set_step_index(s)
        g.step(tdt, 1)
        o.step(tdt, 1)
        e = field_errors(g, o)
        assert e["p"] <= PSI_TOL, "step %d: psi rel L2 %.2e" % (s + 1, e["p"])
        worst = {k: max(worst.get(k, 0.0), v) for k, v in e.items()}
    print("\n" + _row(case, "one step from the oracle's state (max of 3)", worst))
    g.close()
    o.close()
