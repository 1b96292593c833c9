"""The ocean mixed-layer restatement (oracle/mixed_layer.py), pinned by the
properties of the reference's equations (the reference has no tests of this
code) and, for its Ekman part, by the C++ oracle's ekman_from_tau.

  * ekman: wekp within 1e-14 of oracle.ekman_from_tau;
  * adv_diff with no-flux walls conserves heat: its sum over the T cells
    vanishes to rounding (the C-grid fluxes and the del2_T differences
    telescope, and both velocities vanish on the walls);
  * the entrainment's T-grid field has zero mean (omlsubs.F90:110-112);
  * the convective adjustment leaves sst >= T_bar - T_(1) everywhere
    (sstnew + max(0, T1_rel - sstnew), omlsubs.F90:101, 117).
"""
import numpy as np

import oracle
from oracle.mixed_layer import OmlOracle, OmlParams, ekman
from openqg_b200.params import double_gyre_tau, initial_psi, ocean_double_gyre


def _case(n=33, seed=0, **kw):
    b = ocean_double_gyre(n, dx=40.0e3)
    prm = OmlParams(st2d=2.0e3, st4d=1.0e11, ycexp=1.0, **kw)
    o = OmlOracle(b, prm)
    rng = np.random.default_rng(seed)
    nyt, nxt = b.nyp - 1, b.nxp - 1
    yy = np.linspace(0.0, 1.0, nyt)[:, None]
    o.data = prm.t1_rel + 2.0 + 3.0 * np.cos(np.pi * yy) + 0.3 * rng.standard_normal((nyt, nxt))
    o.datam = o.data + 0.05 * rng.standard_normal((nyt, nxt))
    taux, tauy = double_gyre_tau(b)
    tauy = tauy + 0.02 * rng.standard_normal(tauy.shape)
    p1 = b.fnot * initial_psi(b, seed=seed)[0]
    return b, prm, o, taux, tauy, p1, rng


def test_ekman_matches_cpp_oracle():
    b, prm, _, taux, tauy, _, _ = _case()
    _, _, _, wekp = ekman(taux, tauy, b.dx, b.dy, b.fnot, prm.hm)
    w, _, _ = oracle.ekman_from_tau(b, taux, tauy)
    ref = w.reshape(b.shape2)
    assert np.linalg.norm(wekp - ref) <= 1e-14 * np.linalg.norm(ref)


def test_adv_diff_conserves_heat_with_no_flux_walls():
    b, prm, o, taux, tauy, p1, _ = _case()
    uek, vek, _, _ = ekman(taux, tauy, b.dx, b.dy, b.fnot, prm.hm)
    dp_dx = (p1[:, 1:] - p1[:, :-1]) / b.dx
    dp_dy = (p1[1:, :] - p1[:-1, :]) / b.dy
    a = o.adv_diff(dp_dx, dp_dy, uek, vek)
    assert abs(a.sum()) <= 1e-12 * np.abs(a).sum()


def test_entrainment_has_zero_mean_and_sst_is_adjusted():
    b, prm, o, taux, tauy, p1, rng = _case(seed=3)
    uek, vek, wekt, _ = ekman(taux, tauy, b.dx, b.dy, b.fnot, prm.hm)
    fnet = 50.0 * rng.standard_normal(wekt.shape)
    ent = np.ones((b.nl - 1, b.nyp, b.nxp))
    xfo = o.step(p1, uek, vek, wekt, fnet, True, 3600.0, ent)
    assert abs(xfo.sum()) <= 1e-12 * np.abs(xfo).sum()
    assert np.all(ent[1:] == 0.0)
    assert np.all(o.data >= prm.t1_rel)
    # without compute_ent the entrainment is left as it was
    ent2 = ent.copy()
    o.step(p1, uek, vek, wekt, fnet, False, 3600.0, ent2)
    assert np.array_equal(ent2, ent)


# ---------------------------------------------------------------- atmosphere
from oracle.mixed_layer import AmlOracle, AmlParams, adv_diff_cyclic, ekman_cyclic  # noqa: E402
from openqg_b200.params import atmos_channel  # noqa: E402


def _channel_case(seed=0):
    b = atmos_channel(65, 33)
    rng = np.random.default_rng(seed)
    y = np.arange(b.nyp) * b.dy
    taux = np.repeat((0.1 * np.sin(np.pi * y / y[-1]))[:, None], b.nxp, axis=1) + 0.01 * rng.standard_normal(b.shape2)
    tauy = 0.01 * rng.standard_normal(b.shape2)
    taux[:, -1] = taux[:, 0]
    tauy[:, -1] = tauy[:, 0]
    p1 = b.fnot * 30.0 * initial_psi(b, seed=seed)[0]
    return b, rng, taux, tauy, p1


def test_channel_ekman_matches_cpp_oracle():
    b, _, taux, tauy, _ = _channel_case()
    _, _, _, wekp, txis, txin = ekman_cyclic(taux, tauy, b.dx, b.dy, b.fnot, 1000.0)
    w, ts, tn = oracle.ekman_from_tau(b, taux, tauy)
    ref = w.reshape(b.shape2)
    assert np.linalg.norm(wekp - ref) <= 1e-14 * np.linalg.norm(ref)
    assert abs(txis - ts) <= 1e-14 * abs(ts) and abs(txin - tn) <= 1e-14 * abs(tn)


def test_channel_adv_diff_conserves_with_no_flux_walls():
    b, rng, taux, tauy, p1 = _channel_case(1)
    uek, vek, _, _, _, _ = ekman_cyclic(taux, tauy, b.dx, b.dy, b.fnot, 1000.0)
    nyt, nxt = b.nyp - 1, b.nxp - 1
    t = 3.0 * rng.standard_normal((nyt, nxt))
    dp_dx = (p1[:, 1:] - p1[:, :-1]) / b.dx
    dp_dy = (p1[1:, :] - p1[:-1, :]) / b.dy
    a = adv_diff_cyclic(t, t + 0.1, dp_dx, dp_dy, uek, vek, b.fnot, b.dx, b.dy, 2.5e4, 1e12, 1.0,
                        False, False, 0.0, 0.0)
    assert abs(a.sum()) <= 1e-12 * np.abs(a).sum()


def test_atmos_step_bounds():
    """After step_aml the temperature is at most T_bar - T_(1) (the
    convective correction, amlsubs.F90:278-283) and the height at least
    hmamin wherever it was stepped."""
    b, rng, taux, tauy, p1 = _channel_case(2)
    prm = AmlParams(aface=(1e-6, -2e-7), bface=3e-7, dface=1e-5)
    nyt, nxt = b.nyp - 1, b.nxp - 1
    o = AmlOracle(b, prm, xc1ast=0.5 * rng.standard_normal((nyt, nxt)), dtop=np.zeros(b.shape2))
    o.ast = prm.t1_rel - 2.0 + rng.standard_normal((nyt, nxt))
    o.astm = o.ast + 0.1 * rng.standard_normal((nyt, nxt))
    uek, vek, wekt, _, _, _ = ekman_cyclic(taux, tauy, b.dx, b.dy, b.fnot, prm.hm)
    eta = rng.standard_normal((b.nl - 1,) + b.shape2)
    eta[..., -1] = eta[..., 0]          # a channel field repeats column 0
    ent = np.zeros((b.nl - 1,) + b.shape2)
    o.step(p1, uek, vek, wekt, eta, 30.0 * rng.standard_normal((nyt, nxt)), True, 360.0, ent)
    assert np.all(o.ast <= prm.t1_rel)
    assert np.all(o.hmx >= prm.hmamin)
    assert np.array_equal(ent[0][:, -1], ent[0][:, 0]) and np.all(ent[1:] == 0.0)


def test_hermite_bicubic_reproduces_bicubics_and_nodes():
    """The interpolant is exact for a bicubic polynomial given exact scaled
    derivatives, and equals the nodal values at the coarse nodes."""
    from oracle.mixed_layer import hermite_bicubic
    rng = np.random.default_rng(5)
    C = rng.standard_normal((4, 4))
    P = lambda x, y: sum(C[a, c] * x ** a * y ** c for a in range(4) for c in range(4))
    Px = lambda x, y: sum(a * C[a, c] * x ** (a - 1) * y ** c for a in range(1, 4) for c in range(4))
    Py = lambda x, y: sum(c * C[a, c] * x ** a * y ** (c - 1) for a in range(4) for c in range(1, 4))
    Pxy = lambda x, y: sum(a * c * C[a, c] * x ** (a - 1) * y ** (c - 1) for a in range(1, 4) for c in range(1, 4))
    h, nd = 0.3, 6
    X, Y = np.meshgrid(np.arange(5) * h, np.arange(4) * h)
    out = hermite_bicubic(P(X, Y), h * Px(X, Y), h * Py(X, Y), h * h * Pxy(X, Y), nd)
    Xf, Yf = np.meshgrid(np.arange(4 * nd + 1) * h / nd, np.arange(3 * nd + 1) * h / nd)
    ref = P(Xf, Yf)
    assert np.max(np.abs(out - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.array_equal(out[::nd, ::nd], P(X, Y))


# ----------------------------------------------------------- coupled fluxes
from oracle.mixed_layer import RadCoeffs, bilint, compute_forcing, coupling_grid  # noqa: E402


def _pair():
    return ocean_double_gyre(129, dx=10.0e3), atmos_channel(49, 25, dx=80e3)


def test_bilint_reproduces_linear_fields_and_wraps_in_x():
    """Exact for a field linear in x and y where no wrap or end row enters;
    the westmost ocean columns interpolate across the channel's periodic
    seam (the last T column standing half a cell west of the first)."""
    bo, ba = _pair()
    nxta, nyta = ba.nxp - 1, ba.nyp - 1
    _, _, _, c0, r0 = coupling_grid(bo, ba)
    xa = (np.arange(nxta) + 0.5) * ba.dx
    ya = (np.arange(nyta) + 0.5) * ba.dy
    at = 3.0 + 2e-6 * xa[None, :] - 5e-6 * ya[:, None]
    out = bilint(at, bo, ba)
    xo = c0 * ba.dx + (np.arange(bo.nxp - 1) + 0.5) * bo.dx
    yo = r0 * ba.dy + (np.arange(bo.nyp - 1) + 0.5) * bo.dy
    ref = 3.0 + 2e-6 * xo[None, :] - 5e-6 * yo[:, None]
    east = xo >= 0.5 * ba.dx
    assert np.max(np.abs(out[:, east] - ref[:, east])) <= 1e-12
    # the seam: the weights of the last column (at -dx/2) and the first
    w = (xo[~east] + 0.5 * ba.dx) / ba.dx
    seam = (1.0 - w)[None, :] * (3.0 + 2e-6 * xa[-1]) + w[None, :] * (3.0 + 2e-6 * xa[0])
    assert np.max(np.abs(out[:, ~east] - (seam - 5e-6 * yo[:, None]))) <= 1e-12


def test_compute_forcing_budget():
    """With the perturbation, eta, topography and height terms off and
    Dmdown = Dup(0): the ocean's upward fluxes reach the atmosphere times
    the area ratio (summed over its cells), the ocean loses them and gains
    Dmdown times the interpolated temperature; the perturbation forcing
    fsprim sums to zero over the channel's rows."""
    bo, ba = _pair()
    rng = np.random.default_rng(3)
    nyta, nxta = ba.nyp - 1, ba.nxp - 1
    nyto, nxto = bo.nyp - 1, bo.nxp - 1
    astm = -8.0 + rng.standard_normal((nyta, nxta))
    hmxm = np.full((nyta, nxta), 1000.0)
    sstm = 12.0 + rng.standard_normal((nyto, nxto))
    pma = np.zeros((ba.nl, ba.nyp, ba.nxp))
    rad = RadCoeffs(fspco=0.0, xlamda=35.0, d0up=5.5, dmdown=2.5, dup0=2.5, aup00=0.0, adown10=0.0, adown11=0.0)
    fo, fa = compute_forcing(sstm, astm, hmxm, pma, ba, bo, rad, 1000.0, 0.0)
    asto = bilint(astm, bo, ba)
    up = 5.5 * sstm + 35.0 * (sstm - asto)
    assert np.allclose(fo, -2.5 * asto - up, rtol=0, atol=1e-12)
    ocfrac = bo.dx * bo.dy / (ba.dx * ba.dy)
    assert abs(np.sum(fa + 2.5 * astm) - ocfrac * np.sum(up)) <= 1e-9 * np.sum(np.abs(up))
    # only the perturbation forcing: each row constant, rows sum to zero
    rad = RadCoeffs(fspco=80.0, xlamda=0.0, d0up=0.0, dmdown=0.0, dup0=0.0, aup00=0.0, adown10=0.0, adown11=0.0)
    _, fa = compute_forcing(sstm, astm, hmxm, pma, ba, bo, rad, 1000.0, 0.0)
    assert np.allclose(fa, fa[:, :1], rtol=0, atol=1e-12)
    assert abs(np.sum(fa[:, 0])) <= 1e-11 * np.sum(np.abs(fa[:, 0]))


def test_compute_forcing_eta_topography_and_height_terms():
    """The eta_1, topography and height terms alone: T-point averages of
    (pm_1 - pm_2) / gp_1 and dtop scaled by their coefficients, and the
    height damping."""
    bo, ba = _pair()
    rng = np.random.default_rng(4)
    nyta, nxta = ba.nyp - 1, ba.nxp - 1
    pma = rng.standard_normal((ba.nl, ba.nyp, ba.nxp))
    dtop = rng.standard_normal(ba.shape2)
    hmxm = 1000.0 + rng.standard_normal((nyta, nxta))
    rad = RadCoeffs(fspco=0.0, xlamda=0.0, d0up=0.0, dmdown=0.0, dup0=0.0, aup00=-0.03, adown10=0.02, adown11=0.01)
    _, fa = compute_forcing(np.zeros((bo.nyp - 1, bo.nxp - 1)), np.zeros((nyta, nxta)), hmxm, pma, ba, bo, rad,
                            1000.0, 0.5, dtop)
    eta = (pma[0] - pma[1]) / ba.gp[0]
    avg = lambda f: 0.25 * (f[:-1, :-1] + f[:-1, 1:] + f[1:, :-1] + f[1:, 1:])
    ref = -0.01 * avg(eta) - (-0.03 + 0.02) * avg(dtop) + (-0.5 + 0.03 - 0.02) * (hmxm - 1000.0)
    assert np.allclose(fa, ref, rtol=0, atol=1e-12)


def test_tau_udiff_reduces_to_the_atmosphere_alone():
    """With the ocean at rest and an infinitely deep ocean mixed layer the
    velocity-difference stress is the atmosphere-only one; the atmosphere's
    stress over the ocean becomes the ocean-resolution stress before the
    density ratio."""
    from oracle.mixed_layer import atmos_stress, ocean_stress
    bo, ba = _pair()
    rng = np.random.default_rng(6)
    pma = ba.fnot * 1e5 * rng.standard_normal((ba.nyp, ba.nxp))
    pma[:, -1] = pma[:, 0]
    t0 = ocean_stress(pma, ba, bo, 1.3e-3, 1000.0, 1.2e-3)
    t1 = ocean_stress(pma, ba, bo, 1.3e-3, 1000.0, 1.2e-3, pmo1=np.zeros((bo.nyp, bo.nxp)), hmo=np.inf)
    assert np.array_equal(t0[0], t1[0]) and np.array_equal(t0[1], t1[1])
    pmo = bo.fnot * 1e4 * rng.standard_normal((bo.nyp, bo.nxp))
    tax, tay = atmos_stress(pma, ba, 1.3e-3, 1000.0)
    tox, toy = ocean_stress(pma, ba, bo, 1.3e-3, 1000.0, 1.2e-3, pmo1=pmo, hmo=100.0, atmos_tau=(tax, tay))
    ndxr, nxtoar, nytoar, c0, r0 = coupling_grid(bo, ba)
    assert np.allclose(tax[r0:r0 + nytoar + 1, c0:c0 + nxtoar + 1] * 1.2e-3, tox[::ndxr, ::ndxr], rtol=1e-15, atol=0)
    assert not np.allclose(tox, t0[0])
