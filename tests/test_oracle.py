"""Pins of the CPU oracle (no GPU).

The reference has no golden vectors for step_qg, so the oracle is pinned by
the reference's own tests and by properties of the discretisation:
  * src/tests/test_inhomog.F90:18-240 -- Helmholtz residuals, box and channel
    (the sine case run as intended, per point; random cases seeded);
  * src/qg/modes.F90:148-161 -- the mode conversion matrices multiply to I;
  * an O(n^2) long-double DST-I and numpy's FFT for the transforms;
  * energy and enstrophy conservation of the Arakawa Jacobian;
  * mass-constraint closure after box_homog (homog.F90:331-366);
  * an independent numpy reading of qcomp (vorsubs.F90:27-56).
"""
import numpy as np
import pytest

import oracle
from openqg_b200.params import (Basin, atmos_channel, double_gyre_tau,
                                initial_psi, ocean_double_gyre)
from tests import qg_numpy as qn


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 15, 30, 63, 79, 95, 127, 191, 255, 511])
def test_dst1_matches_long_double_direct(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    fast = oracle.dst1(x[None, :])[0]
    ref = oracle.dst1_direct(x)
    assert np.abs(fast - ref).max() <= 2e-15 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("N", [4, 12, 96, 100, 192, 384])
def test_rfft_matches_numpy_and_roundtrips(N):
    rng = np.random.default_rng(N)
    x = rng.standard_normal((5, N))
    X = oracle.rfft(x)
    assert np.abs(X - np.fft.rfft(x)).max() <= 1e-14 * np.abs(X).max()
    back = oracle.irfft(X, N) / N
    assert np.abs(back - x).max() <= 1e-14


def _test_box(cyclic):
    # test_inhomog.F90:26-53: 100x100 10 km channel; 80x100 box
    if cyclic:
        return Basin(nxp=101, nyp=101, dx=1e4, dy=1e4, h=[1000.0, 2000.0, 3000.0],
                     gp=[0.02, 0.01], cyclic=True, dz_sign=1)
    return Basin(nxp=81, nyp=101, dx=1e4, dy=1e4, h=[1000.0, 2000.0, 3000.0],
                 gp=[0.02, 0.01], cyclic=False, dz_sign=1)


RDM2 = np.array([0.0, 1.0 / 50000.0 ** 2, 1.0 / 150000.0 ** 2])   # test_inhomog.F90:34


def _rhs_cases(b, seed):
    nyp, nxp = b.shape2
    i = np.arange(1, nxp + 1)[None, :]
    j = np.arange(1, nyp + 1)[:, None]
    cases = {
        "constant": np.ones(b.shape2),
        # the reference loop (test_inhomog.F90:95-99) assigns the whole array
        # each pass, so its "sine" case is this constant:
        "sine_as_coded": np.full(b.shape2, 2.0 * np.sin(5.0) + 3.0 * np.sin(2.0)),
        "sine": 2.0 * np.sin(5.0 * i / nxp) + 3.0 * np.sin(2.0 * j / nyp),
        "random": np.random.default_rng(seed).random(b.shape2),
    }
    if b.cyclic:
        for v in cases.values():
            v[:, -1] = v[:, 0]
    return cases


@pytest.mark.parametrize("cyclic", [False, True])
def test_inhomog_residual_reference_cases(cyclic):
    """test_rhs, test_inhomog.F90:123-154: residual <= 1e-11 (relative)."""
    b = _test_box(cyclic)
    o = oracle.Oracle(b)
    o.set_rdm2(RDM2)
    for name, rhs in _rhs_cases(b, 7).items():
        for m in (1, 2, 3):
            soln = o.solve_inhomog(m, rhs)
            out = o.del2(soln, 0.0) - RDM2[m - 1] * soln
            sl = (slice(1, -1), slice(None)) if cyclic else (slice(1, -1), slice(1, -1))
            res = np.abs(out[sl] - rhs[sl]).max() / np.abs(rhs[sl]).max()
            assert res <= 1e-11, (name, m, res)
            # boundary conditions of the solver
            assert np.all(soln[0, :] == 0) and np.all(soln[-1, :] == 0)
            if cyclic:
                assert np.array_equal(soln[:, -1], soln[:, 0])
            else:
                assert np.all(soln[:, 0] == 0) and np.all(soln[:, -1] == 0)


@pytest.mark.parametrize("cyclic", [False, True])
def test_homog_residual_reference_cases(cyclic):
    """test_L, test_inhomog.F90:208-240: (Del2 - rdm2) soln == Del2 L.

    The reference threshold is 1e-22 relative to max|L|; the residual of
    generate_homog_soln is rdm2 times the Helmholtz residual, so it is tiny.
    """
    b = _test_box(cyclic)
    o = oracle.Oracle(b)
    o.set_rdm2(RDM2)
    for name, L in _rhs_cases(b, 11).items():
        for m in (1, 2, 3):
            soln = o.generate_homog_soln(m, L)
            out1 = o.del2(soln, 0.0) - RDM2[m - 1] * soln
            out2 = o.del2(L, 0.0)
            sl = (slice(1, -1), slice(None)) if cyclic else (slice(1, -1), slice(1, -1))
            res = np.abs(out1[sl] - out2[sl]).max() / np.abs(L[sl]).max()
            assert res <= 1e-22, (name, m, res)


@pytest.mark.parametrize("basin", [ocean_double_gyre(65), atmos_channel(33, 17)])
def test_modes_identity_and_eigen(basin):
    """ccprod check (modes.F90:148-161) and A R = lambda R."""
    o = oracle.Oracle(basin)
    md = o.modes()
    cm2l, cl2m = md["ctm2l"].T, md["ctl2m"].T
    assert np.abs(cm2l @ cl2m - np.eye(basin.nl)).max() <= 5e-15
    assert md["rdm2"][0] == 0.0
    lam = md["rdm2"] / basin.fnot ** 2
    A = md["amat"]
    for m in range(basin.nl):
        r = cm2l[:, m]
        assert np.abs(A @ r - lam[m] * r).max() <= 1e-12 * np.abs(A).max() * np.abs(r).max()
    # compute_A, modes.F90:221-246
    h, g = basin.h, basin.gp
    assert A[0, 1] == -1.0 / (g[0] * h[0]) and A[0, 0] == -A[0, 1]
    assert np.all(np.diff(md["rdm2"]) > 0)


def test_jacobian_conservation():
    """Arakawa: sum p J(q,p) = 0 and sum q J(q,p) = 0 (p, q zero on walls)."""
    b = ocean_double_gyre(65)
    o = oracle.Oracle(b)
    rng = np.random.default_rng(3)
    p = np.zeros(b.shape2)
    q = np.zeros(b.shape2)
    p[1:-1, 1:-1] = rng.standard_normal((63, 63))
    q[1:-1, 1:-1] = rng.standard_normal((63, 63))
    J = o.jacobian(p, q)
    scale = np.abs(J * p).sum()
    assert abs((J * p).sum()) <= 1e-13 * scale
    assert abs((J * q).sum()) <= 1e-13 * np.abs(J * q).sum()
    # an independent numpy reading of the same stencil
    Jn = qn.jacobian(p, q, b.dx, b.dy, b.fnot, False)
    assert np.abs(J - Jn).max() <= 1e-14 * np.abs(Jn).max()


@pytest.mark.parametrize("basin", [ocean_double_gyre(33), atmos_channel(33, 17)])
def test_init_pv_matches_numpy(basin):
    o = oracle.Oracle(basin)
    p = basin.fnot * initial_psi(basin, seed=5)
    pm = basin.fnot * initial_psi(basin, seed=6)
    o.set_state(p, pm)
    _, _, q, qm = o.get_state()
    A = o.modes()["amat"]
    assert qn.rel_l2(q, qn.qcomp(p, A, basin)) <= 1e-14
    assert qn.rel_l2(qm, qn.qcomp(pm, A, basin)) <= 1e-14


def test_mass_constraint_closure_box():
    """After box_homog, int (p_{k+1} - p_k) dA == dpi_k (homog.F90:331-366)."""
    b = ocean_double_gyre(65)
    o = oracle.Oracle(b)
    p = b.fnot * initial_psi(b, seed=2)
    o.set_state(p, p)
    taux, tauy = double_gyre_tau(b)
    w, _, _ = oracle.ekman_from_tau(b, taux, tauy)
    o.set_forcing(w)
    for _ in range(5):
        o.step(3600.0, 1)
        P = o.get_state()[0]
        dpi = o.get_constraints()["dpi"]
        ints = np.array([o.int_P_dA(P[k]) for k in range(b.nl)])
        diff = ints[1:] - ints[:-1]
        assert np.allclose(diff, dpi, rtol=0, atol=1e-10 * np.abs(ints).max())


def test_suppress_schedule_matches_explicit_average():
    """mod(nt-1, period) == 0 applies suppress_comp_mode after step nt."""
    b = ocean_double_gyre(33)
    p = b.fnot * initial_psi(b, seed=4)
    A = oracle.Oracle(b)                       # period 25 (default)
    b0 = ocean_double_gyre(33, suppress_period=0)
    B = oracle.Oracle(b0)
    for o in (A, B):
        o.set_state(p, p)
        o.set_forcing(None)
    A.step(3600.0, 2)
    B.step(3600.0, 1)
    B.suppress()
    B.step(3600.0, 1)
    for x, y in zip(A.get_state(), B.get_state()):
        assert np.array_equal(x, y)


def test_ekman_double_gyre_curl():
    """wekp of the analytic stress approximates -(1/f0) d(tau_x)/dy."""
    b = ocean_double_gyre(129)
    taux, tauy = double_gyre_tau(b)
    w, txis, txin = oracle.ekman_from_tau(b, taux, tauy)
    yl = (b.nyp - 1) * b.dy
    y = np.arange(b.nyp) * b.dy
    exact = -(0.1 / 1e3) * (2 * np.pi / yl) * np.sin(2 * np.pi * y / yl) / b.fnot
    err = np.abs(w[1:-1, 1:-1] - exact[1:-1, None]).max() / np.abs(exact).max()
    assert err < 1e-3
    assert txis == 0.0 and txin == 0.0


def test_channel_steps_finite_and_periodic():
    b = atmos_channel(49, 25)
    o = oracle.Oracle(b)
    p = b.fnot * initial_psi(b, seed=8) * 50.0
    o.set_state(p, p)
    o.set_forcing(None)
    o.step(360.0, 20)
    P, PM, Q, QM = o.get_state()
    assert np.isfinite(P).all() and np.isfinite(Q).all()
    assert np.array_equal(P[:, :, -1], P[:, :, 0])


def test_diagno_record_consistent():
    """The oracle's qg_diagno: its ekei is diag's, the double-gyre pumping
    averages to zero, the energy rate pket follows from two calls, and
    ctot sums circ."""
    b = ocean_double_gyre(33)
    o = oracle.Oracle(b)
    p = b.fnot * initial_psi(b, 1)
    o.set_state(p, p)
    taux, tauy = double_gyre_tau(b)
    w, ts, tn = oracle.ekman_from_tau(b, taux, tauy)
    o.set_forcing(w, None, ts, tn)
    o.step(3600.0, 3)
    d1, mon = o.diagno(taux, tauy, tsec=100.0, tdt=3600.0)
    assert np.allclose(d1["ekei"], o.diag()["ekei"], rtol=1e-12)
    assert abs(d1["wepm"]) <= 1e-10 * d1["wapm"]
    assert d1["ctot"] == pytest.approx(np.sum(d1["circ"]))
    et2_first = d1["et2m"].copy()
    o.step(3600.0, 1)
    d2, _ = o.diagno(taux, tauy, tsec=3700.0, tdt=3600.0, mon=mon)
    want = 0.5 * b.rho * np.array(b.gp) * (d2["et2m"] - et2_first) / 3600.0
    assert np.allclose(d2["pket"], want, rtol=1e-12)
