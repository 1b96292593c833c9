"""The committed golden step fixtures (tests/golden, made by make_golden.py
from the FP64 oracle on seeded inputs).

CPU: the oracle as built here still reproduces them.  GPU: the CUDA path,
through the C ABI, matches them with the parity tolerances (relative L2:
1e-12 after 1 step, 1e-10 after 10 steps).
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402
import oracle  # noqa: E402
from tests.qg_numpy import rel_l2  # noqa: E402

NAMES = sorted(make_golden.CASES)


def _load(name):
    return dict(np.load(os.path.join(HERE, "golden", "golden_%s.npz" % name)))


def _basin(name):
    return make_golden.CASES[name][0]()


def _run(x, g):
    g.set_state(x["p0"], x["pm0"])
    g.set_forcing(x["wekp"], x.get("ent"), float(x["txis"]), float(x["txin"]))
    tdt = float(x["tdt"])
    g.step(tdt, 1)
    p1, _, q1, _ = g.get_state()
    g.step(tdt, 9)
    p10, _, q10, _ = g.get_state()
    return p1, q1, p10, q10


@pytest.mark.parametrize("name", NAMES)
def test_inputs_regenerate_from_seeds(name):
    b, tdt, p, pm, wekp, ent, txis, txin = make_golden.inputs(name)
    x = _load(name)
    assert np.array_equal(x["p0"], p) and np.array_equal(x["pm0"], pm)
    assert rel_l2(wekp, x["wekp"]) <= 1e-15
    if ent is not None:
        assert np.array_equal(x["ent"], ent)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(name):
    x = _load(name)
    o = oracle.Oracle(_basin(name))
    p1, q1, p10, q10 = _run(x, o)
    for a, key in ((p1, "p1"), (q1, "q1"), (p10, "p10"), (q10, "q10")):
        assert rel_l2(a, x[key]) <= 1e-13, key


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_cuda_step_matches_golden(name, gpu_required):
    from openqg_b200.core import QG
    x = _load(name)
    g = QG(_basin(name))
    p1, q1, p10, q10 = _run(x, g)
    assert rel_l2(p1, x["p1"]) <= 1e-12 and rel_l2(q1, x["q1"]) <= 1e-12
    assert rel_l2(p10, x["p10"]) <= 1e-10 and rel_l2(q10, x["q10"]) <= 1e-10
    dpi = g.constraints()["dpi"]
    assert np.allclose(dpi, x["dpi10"], rtol=1e-9, atol=1e-9 * np.abs(x["dpi10"]).max())
    g.close()
