"""Batched ensembles (oqg_ensemble_*): members of uneven size stepped by one
launch per phase must give what each member gives as a single handle (to
rounding), and so inherit the single handle's parity with the oracle."""
import numpy as np
import pytest

import oracle
from openqg_b200.core import QG, Ensemble
from openqg_b200.params import OQG_MIXED, atmos_channel, double_gyre_tau, initial_psi, ocean_double_gyre
from tests.qg_numpy import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu(gpu_required):
    pass


def _channel_tau(b, amp=0.1):
    yl = (b.nyp - 1) * b.dy
    y = np.arange(b.nyp) * b.dy
    taux = np.repeat((amp * np.sin(np.pi * y / yl))[:, None], b.nxp, axis=1)
    return taux, np.zeros_like(taux)


def _inputs(b, seed):
    amp = 30.0 if b.cyclic else 1.0
    p = b.fnot * initial_psi(b, seed) * amp
    pm = 0.5 * p + 0.25 * b.fnot * initial_psi(b, seed + 11) * amp
    taux, tauy = _channel_tau(b, 0.05 + 0.02 * seed) if b.cyclic else double_gyre_tau(b)
    if not b.cyclic:
        taux = taux * (0.5 + 0.25 * seed)
    return p, pm, oracle.ekman_from_tau(b, taux, tauy)


def _run_pair(members, tdts, nsteps):
    e = Ensemble(members)
    singles = []
    for i, b in enumerate(members):
        p, pm, (w, ts, tn) = _inputs(b, i + 1)
        e.set_state(i, p, pm)
        e.set_forcing(i, w, None, ts, tn)
        g = QG(b)
        g.set_state(p, pm)
        g.set_forcing(w, None, ts, tn)
        singles.append(g)
    e.step(tdts, nsteps)
    e.sync()
    for g, t in zip(singles, np.broadcast_to(tdts, (len(members),))):
        g.step(float(t), nsteps)
    return e, singles


def _assert_same(e, singles, tol=1e-13):
    # members tile the vorticity kernel with the tallest (or a tuned) height, single handles
    # with tiles fitted to whole waves; the channel strip sums and the wall
    # rows then round differently, so the match is to rounding, not bits
    # (FP64 rounding; FP32 storage rounds at about 1e-7)
    for i, g in enumerate(singles):
        for name, a, c in zip(("p", "pm", "q", "qm"), e.get_state(i), g.get_state()):
            assert rel_l2(a, c) <= tol, "member %d %s rel L2 %.3e" % (i, name, rel_l2(a, c))


def test_box_ensemble_equals_single_handles():
    members = [ocean_double_gyre(n) for n in (65, 129, 33, 97)]
    members[1].ah4 = [3e10] * 3
    e, singles = _run_pair(members, 3600.0, 5)      # 2 graph replays + 1 launch
    _assert_same(e, singles)
    e.step(3600.0, 3)
    for g in singles:
        g.step(3600.0, 3)
    _assert_same(e, singles)


def test_uniform_box_ensemble_equals_single_handles():
    """Members of one transform length take that length's transform
    instances, as a single handle of the same size does."""
    members = [ocean_double_gyre(129) for _ in range(3)]
    for i, b in enumerate(members):
        b.ah4 = [(1.0 + i) * 1e10] * 3
    e, singles = _run_pair(members, 3600.0, 4)
    _assert_same(e, singles)


def test_box_ensemble_member_matches_oracle():
    members = [ocean_double_gyre(97), ocean_double_gyre(65)]
    e = Ensemble(members)
    orc = []
    for i, b in enumerate(members):
        p, pm, (w, ts, tn) = _inputs(b, i + 1)
        e.set_state(i, p, pm)
        e.set_forcing(i, w, None, ts, tn)
        o = oracle.Oracle(b)
        o.set_state(p, pm)
        o.set_forcing(w, None, ts, tn)
        orc.append(o)
    e.step(3600.0, 10)
    for o in orc:
        o.step(3600.0, 10)
    for i, o in enumerate(orc):
        for name, a, c in zip(("p", "q"), e.get_state(i)[::2], o.get_state()[::2]):
            assert rel_l2(a, c) <= 1e-10, (i, name)


def test_channel_ensemble_equals_single_handles():
    members = [atmos_channel(49, 25), atmos_channel(97, 65), atmos_channel(193, 97)]
    e, singles = _run_pair(members, 360.0, 4)
    _assert_same(e, singles)


def test_per_member_step_and_mixed_precision():
    members = [ocean_double_gyre(n, precision=OQG_MIXED) for n in (129, 65, 97)]
    tdts = np.array([3600.0, 1800.0, 2400.0])
    e, singles = _run_pair(members, tdts, 4)
    _assert_same(e, singles, tol=1e-6)


def test_ensemble_rejects_bad_members():
    from openqg_b200.core import OqgError
    with pytest.raises(OqgError):
        Ensemble([ocean_double_gyre(33), atmos_channel(49, 25)])


def test_ensemble_autotune_keeps_states_and_results():
    """oqg_ensemble_autotune retiles every member to the measured height; the
    members' states are restored, and stepping on matches single handles."""
    members = [ocean_double_gyre(n, dx=20e3) for n in (129, 65, 97)]
    e, singles = _run_pair(members, 3600.0, 2)
    before = [e.get_state(i) for i in range(len(members))]
    best, ms = e.autotune(3600.0, 4)
    assert best in (8, 12, 16)
    assert sorted(ms) == [8, 12, 16]
    for i in range(len(members)):
        for a, r in zip(e.get_state(i), before[i]):
            assert np.array_equal(a, r)
    e.step(3600.0, 6)
    e.sync()
    for g in singles:
        g.step(3600.0, 6)
    _assert_same(e, singles)
