"""The tile-height autotuner (oqg_autotune): it measures every height on the
device, keeps the fastest, leaves the state as it found it, and later handles
of the same shape start from the measured height.  Stepping with the tuned
tiles matches stepping with the default ones within 1e-12 relative L2 (the
tiles change where a point is computed, not how; rounding may differ in the
order of the wall terms' operations)."""
import numpy as np
import pytest

import oracle
from openqg_b200.core import QG, OqgError
from openqg_b200.params import OQG_MIXED, atmos_channel, double_gyre_tau, initial_psi, ocean_double_gyre
from tests.qg_numpy import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu(gpu_required):
    pass


def _handle(b, seed=1):
    g = QG(b)
    p = b.fnot * initial_psi(b, seed=seed) * (30.0 if b.cyclic else 1.0)
    if b.cyclic:
        y = np.arange(b.nyp) * b.dy
        taux = np.repeat((0.05 * np.sin(np.pi * y / y[-1]))[:, None], b.nxp, axis=1)
        w, ts, tn = oracle.ekman_from_tau(b, taux, np.zeros_like(taux))
    else:
        w, ts, tn = oracle.ekman_from_tau(b, *double_gyre_tau(b))
    g.set_state(p, p)
    g.set_forcing(w, None, ts, tn)
    return g


@pytest.mark.parametrize("precision,channel", [(0, False), (OQG_MIXED, False), (0, True)])
def test_autotune_keeps_state_and_results(precision, channel):
    """Box (tiles by TMA) in FP64 and mixed; channel (tiles by cp.async, strip
    sums over the tiles of the boundary rows)."""
    b = (atmos_channel(193, 97, precision=precision) if channel
         else ocean_double_gyre(161, dx=20e3, precision=precision))
    g, ref = _handle(b), _handle(b)
    tdt = 360.0 if channel else 3600.0
    g.step(tdt, 3)
    ref.step(tdt, 3)
    before = g.get_state()
    best, ms = g.autotune(tdt, 6)
    assert best in (8, 12, 16) and g.tile_rows() == best
    assert sorted(ms) == [8, 12, 16] and all(v > 0 for v in ms.values())
    for a, r in zip(g.get_state(), before):
        assert np.array_equal(a, r)
    assert g.step_index() == 3
    g.step(tdt, 5)
    ref.step(tdt, 5)
    tol = 1e-12 if precision == 0 else 1e-6
    for a, r in zip(g.get_state(), ref.get_state()):
        assert rel_l2(a, r) <= tol
    # a new handle of the same shape and precision starts from the tuned height
    g2 = QG(b)
    assert g2.tile_rows() == best
    for x in (g, ref, g2):
        x.close()


@pytest.mark.parametrize("n,channel", [(257, False), (161, True)])
def test_ysolve_warps_tuning_keeps_state_and_results(n, channel):
    """The y-solve with 1, 2 and 4 warps per column: the tuner times each,
    keeps the fastest, leaves the state as found, and stepping with the
    chosen split matches the default one to rounding."""
    b = atmos_channel(n, 97) if channel else ocean_double_gyre(n)
    g, ref = _handle(b), _handle(b)
    tdt = 360.0 if channel else 3600.0
    g.step(tdt, 2)
    ref.step(tdt, 2)
    before = g.get_state()
    w0 = g.ysolve_warps()
    assert w0 in (1, 2, 4)
    best, ms = g.autotune_ysolve(tdt, 4)
    assert best in (1, 2, 4) and g.ysolve_warps() == best
    assert sorted(ms) == [1, 2, 4] and all(v > 0 for v in ms.values())
    for a, r in zip(g.get_state(), before):
        assert np.array_equal(a, r)
    g.step(tdt, 5)
    ref.step(tdt, 5)
    for a, r in zip(g.get_state(), ref.get_state()):
        assert rel_l2(a, r) <= 1e-12
    for x in (g, ref):
        x.close()


def test_fixed_settings_are_kept_and_checked():
    b = ocean_double_gyre(129)
    g, ref = _handle(b), _handle(b)
    g.set_tile_rows(12)
    g.set_ysolve_warps(4)
    assert g.tile_rows() == 12 and g.ysolve_warps() == 4
    for bad in (lambda: g.set_tile_rows(10), lambda: g.set_ysolve_warps(3)):
        with pytest.raises(OqgError):
            bad()
    g.step(3600.0, 4)
    ref.step(3600.0, 4)
    for a, r in zip(g.get_state(), ref.get_state()):
        assert rel_l2(a, r) <= 1e-12
    for x in (g, ref):
        x.close()


def test_inverse_form_tuning_keeps_state_and_results():
    """A box below 1025 points: the tuner times the one-kernel and the
    two-launch inverse, keeps the faster, leaves the state as found, and
    steps match the default form's to rounding."""
    b = ocean_double_gyre(129)
    g, ref = _handle(b), _handle(b)
    g.step(3600.0, 2)
    ref.step(3600.0, 2)
    before = g.get_state()
    best, ms = g.autotune_xinv(3600.0, 4)
    assert g.xinv_sep() == best
    assert sorted(ms) == [False, True] and all(v > 0 for v in ms.values())
    for a, r in zip(g.get_state(), before):
        assert np.array_equal(a, r)
    g.step(3600.0, 5)
    ref.step(3600.0, 5)
    for a, r in zip(g.get_state(), ref.get_state()):
        assert rel_l2(a, r) <= 1e-12
    for x in (g, ref):
        x.close()
