"""The hand-written adjoint (oqg_adj_*) against a plain-PyTorch autograd
restatement of the step (oracle/torch_step.py) and central finite
differences.

Tolerances:
  * one reversed step and the transpose of set_state: every adjoint output
    within 1e-10 relative L2 of torch autograd's vector-Jacobian product
    (the two differ by rounding only; the Helmholtz solves differ in method);
  * a checkpointed multi-step run: the gradients within 1e-9 of autograd
    through the same number of restated steps;
  * central finite differences (eps = 1e-4 relative) along seeded random
    directions: within 1e-6 relative of the directional derivative.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle
from oracle.torch_step import TorchBox
from openqg_b200.adjoint import AdjointRun, QGRun, ekei
from openqg_b200.core import QG, _check, lib
from openqg_b200.params import OQG_MIXED, atmos_channel, double_gyre_tau, initial_psi, ocean_double_gyre
from tests.qg_numpy import rel_l2

pytestmark = pytest.mark.gpu

TDT = 3600.0


@pytest.fixture(autouse=True)
def _need_gpu(gpu_required):
    pass


def _basin(n=33, nl=3):
    b = ocean_double_gyre(n, dx=40.0e3, ah4=2.0e11)
    b.ah2 = [300.0, 200.0, 100.0]   # exercise the Laplacian friction too
    if nl == 2:
        b.h, b.gp, b.ah2, b.ah4 = [1000.0, 3000.0], [0.02], [300.0, 100.0], [2.0e11] * 2
    elif nl == 4:
        b.h, b.gp = [300.0, 500.0, 800.0, 2400.0], [0.04, 0.02, 0.01]
        b.ah2, b.ah4 = [300.0, 200.0, 150.0, 100.0], [2.0e11] * 4
    return b


def _forcing(b):
    tx, ty = double_gyre_tau(b)
    w, _, _ = oracle.ekman_from_tau(b, tx, ty)
    return w.reshape(b.shape2)


def _state(b, g, nsteps=2, seed=1):
    """A handle advanced a few steps from a seeded start, and its state."""
    p = b.fnot * initial_psi(b, seed=seed)
    pm = p + 0.05 * b.fnot * initial_psi(b, seed=seed + 5)
    g.set_state(p, pm)
    g.set_forcing(_forcing(b), None, 0.0, 0.0)
    g.step(TDT, nsteps)
    g.sync()
    p, pm, q, qm = g.get_state()
    c = g.constraints()
    return [p, pm, q, qm, c["dpi"], c["dpip"]]


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@pytest.mark.parametrize("step_no,nl", [(1, 3), (2, 3), (2, 2), (2, 4)])
def test_one_step_vjp_matches_autograd(step_no, nl):
    """step_no 1 is followed by suppress_comp_mode (period 25), step 2 is not;
    nl 2 and 4 take the transposed constraint solve with 1 and 3 unknowns."""
    b = _basin(nl=nl)
    g, o = QG(b), oracle.Oracle(b)
    st = _state(b, g)
    wekp = _forcing(b)
    tb = TorchBox(b, o)
    xs = [torch.tensor(a, dtype=torch.float64, requires_grad=True) for a in st]
    w = torch.tensor(wekp, dtype=torch.float64, requires_grad=True)
    out = tb.step(*xs, w, TDT, suppress=(step_no - 1) % b.suppress_period == 0)
    rng = np.random.default_rng(10 + step_no)
    cot = [rng.standard_normal(t.shape) * (1.0 / max(float(np.abs(t.detach().numpy()).max()), 1e-30)) for t in out]
    grads = torch.autograd.grad(out, xs + [w], [torch.tensor(c) for c in cot])
    # the device: the handle already holds this state (p, q are the input)
    dev = torch.device("cuda")
    seeds = [torch.tensor(c, dtype=torch.float64, device=dev).contiguous() for c in cot[:4]]
    L = lib()
    torch.cuda.synchronize()
    _check(L.oqg_adj_set(g.h, *[_ptr(s) for s in seeds], _dp(np.ascontiguousarray(cot[4])),
                         _dp(np.ascontiguousarray(cot[5]))), "adj_set")
    run = AdjointRun(g, every=1)
    _check(L.oqg_pq_save(g.h, _ptr(run.slots[0])), "pq_save")
    _check(L.oqg_adj_step(g.h, _ptr(run.slots[0]), ctypes.c_double(TDT), ctypes.c_longlong(step_no)), "adj_step")
    res = [np.empty(b.shape3) for _ in range(4)] + [np.empty(b.nl - 1), np.empty(b.nl - 1), np.empty(b.shape2)]
    _check(L.oqg_adj_get(g.h, *[ctypes.c_void_p(r.ctypes.data) for r in res[:4]], _dp(res[4]), _dp(res[5]),
                         ctypes.c_void_p(res[6].ctypes.data)), "adj_get")
    names = ["p", "pm", "q", "qm", "dpi", "dpip", "wekp"]
    for name, a, r in zip(names, res, grads):
        r = r.numpy()
        err = rel_l2(a, r)
        assert err <= 1e-10, "lambda_%s: rel L2 %.3e" % (name, err)
    g.close()


def test_initial_transpose_matches_autograd():
    b = _basin()
    g, o = QG(b), oracle.Oracle(b)
    tb = TorchBox(b, o)
    p = b.fnot * initial_psi(b, seed=4)
    pm = p + 0.1 * b.fnot * initial_psi(b, seed=9)
    xp = torch.tensor(p, requires_grad=True)
    xpm = torch.tensor(pm, requires_grad=True)
    out = tb.init_state(xp, xpm)
    rng = np.random.default_rng(3)
    cot = [rng.standard_normal(t.shape) for t in out]
    gp, gpm = torch.autograd.grad(out, [xp, xpm], [torch.tensor(c) for c in cot])
    L = lib()
    _check(L.oqg_adj_set(g.h, *[ctypes.c_void_p(np.ascontiguousarray(c).ctypes.data) for c in cot[:4]],
                         _dp(np.ascontiguousarray(cot[4])), _dp(np.ascontiguousarray(cot[5]))), "adj_set")
    a, am = np.empty(b.shape3), np.empty(b.shape3)
    _check(L.oqg_adj_initial(g.h, ctypes.c_void_p(a.ctypes.data), ctypes.c_void_p(am.ctypes.data)), "adj_initial")
    assert rel_l2(a, gp.numpy()) <= 1e-10
    assert rel_l2(am, gpm.numpy()) <= 1e-10
    g.close()


def _objective(b, p):
    return ekei(b, p)[0]


def test_checkpointed_run_matches_autograd_through_steps():
    """12 steps, checkpoints every 5 (segments of 5, 5, 2), suppression at
    step 1: the device gradient against autograd through 12 restated steps."""
    b = _basin()
    b.suppress_period = 10          # suppression after steps 1 and 11
    o = oracle.Oracle(b)
    tb = TorchBox(b, o)
    psi = torch.tensor(initial_psi(b, seed=2), dtype=torch.float64, requires_grad=True)
    curl = torch.tensor(b.fnot * _forcing(b), dtype=torch.float64, requires_grad=True)
    n = 12
    st = tb.init_state(b.fnot * psi, b.fnot * psi)
    for s in range(1, n + 1):
        st = tb.step(*st, curl / b.fnot, TDT, suppress=(s - 1) % b.suppress_period == 0)
    J = _objective(b, st[0])
    gpsi, gcurl = torch.autograd.grad(J, [psi, curl])
    g = QG(b)
    dpsi = psi.detach().cuda().requires_grad_(True)
    dcurl = curl.detach().cuda().requires_grad_(True)
    pf = QGRun.apply(dpsi, dcurl, g, n, TDT, 5)
    Jd = _objective(b, pf)
    assert abs(float(Jd.detach()) - float(J.detach())) <= 1e-12 * abs(float(J.detach()))
    Jd.backward()
    assert rel_l2(dpsi.grad.cpu().numpy(), gpsi.numpy()) <= 1e-9
    assert rel_l2(dcurl.grad.cpu().numpy(), gcurl.numpy()) <= 1e-9
    g.close()


def test_gradient_matches_central_differences():
    """40 steps with checkpoints every 8, J = ekei(1) of the final state;
    central differences along 8 seeded random directions of (psi0, curl)."""
    b = _basin()
    g = QG(b)
    n, every = 40, 8
    psi0 = torch.tensor(initial_psi(b, seed=6), dtype=torch.float64, device="cuda")
    curl0 = torch.tensor(b.fnot * _forcing(b), dtype=torch.float32, device="cuda")

    def J(psi, curl):
        with torch.no_grad():
            return float(_objective(b, QGRun.apply(psi, curl, g, n, TDT, every)))

    psi = psi0.clone().requires_grad_(True)
    curl = curl0.clone().requires_grad_(True)
    Jv = _objective(b, QGRun.apply(psi, curl, g, n, TDT, every))
    Jv.backward()
    gpsi, gcurl = psi.grad.double(), curl.grad.double()
    rng = np.random.default_rng(21)
    for d in range(8):
        dp = torch.tensor(rng.standard_normal(b.shape3), device="cuda")
        dp[:, [0, -1], :] = 0.0
        dp[:, :, [0, -1]] = 0.0
        if d % 2 == 0:
            dc = torch.zeros_like(curl0, dtype=torch.float64)
        else:
            dc = torch.tensor(rng.standard_normal(b.shape2), device="cuda")
        eps_p = 1e-4 * float(psi0.norm()) / float(dp.norm())
        # the curl control is FP32: its finite difference steps along the
        # direction at FP32-representable size; J's FP64 run takes it exactly
        eps_c = 0.0 if d % 2 == 0 else 1e-4 * float(curl0.double().norm()) / float(dc.norm())
        cp = (curl0.double() + eps_c * dc).float()
        cm = (curl0.double() - eps_c * dc).float()
        fd = (J(psi0 + eps_p * dp, cp) - J(psi0 - eps_p * dp, cm)) / 2.0
        dcp = (cp.double() - cm.double()) / 2.0
        an = eps_p * float((gpsi * dp).sum()) + float((gcurl * dcp).sum())
        assert abs(fd - an) <= 1e-6 * abs(an), "direction %d: fd %.12e adjoint %.12e" % (d, fd, an)
    g.close()


def test_adjoint_rejects_channel_and_mixed():
    for b in (atmos_channel(33, 17), ocean_double_gyre(33, precision=OQG_MIXED)):
        g = QG(b)
        rc = lib().oqg_adj_set(g.h, None, None, None, None, None, None)
        assert rc == 5   # OQG_EUNSUPPORTED
        with pytest.raises(ValueError):
            AdjointRun(g)
        g.close()


def test_state_slots_round_trip():
    """state_save / state_load continue bit for bit; pq_save holds p and q."""
    b = _basin()
    g = QG(b)
    _state(b, g, nsteps=3)
    run = AdjointRun(g, every=2)
    slot = torch.empty(run.full_bytes, dtype=torch.uint8, device="cuda")
    _check(lib().oqg_state_save(g.h, _ptr(slot)), "save")
    g.step(TDT, 5)
    a = g.get_state()
    _check(lib().oqg_state_load(g.h, _ptr(slot)), "load")
    g.step(TDT, 5)
    for x, y in zip(a, g.get_state()):
        assert np.array_equal(x, y)
    pq = run.slots[0]
    _check(lib().oqg_pq_save(g.h, _ptr(pq)), "pq_save")
    g.sync()
    p, _, q, _ = g.get_state()
    nb = run.pq_bytes
    f = pq.cpu().numpy().view(np.float64)
    px = (b.nxp + 31) // 32 * 32
    n3 = b.nl * b.nyp * px
    fp = f[:n3].reshape(b.nl, b.nyp, px)[:, :, :b.nxp]
    fq = f[n3:2 * n3].reshape(b.nl, b.nyp, px)[:, :, :b.nxp]
    assert np.array_equal(fp, p) and np.array_equal(fq, q)
    assert nb >= 2 * n3 * 8
    g.close()


def test_one_step_vjp_eddy_resolving_box():
    """The eddy-resolving box (2049x2049x3, dx 5 km, ah4 1e9; its rows are
    wide enough for the split-mode inverse transform): one reversed step
    against autograd through the restated step, run by torch on the GPU."""
    b = ocean_double_gyre(2049, dx=5.0e3, ah4=1.0e9)
    g, o = QG(b), oracle.Oracle(b)
    st = _state(b, g, nsteps=2, seed=3)
    wekp = _forcing(b)
    dev = torch.device("cuda")
    tb = TorchBox(b, o, device=dev)
    xs = [torch.tensor(a, dtype=torch.float64, device=dev, requires_grad=True) for a in st]
    w = torch.tensor(wekp, dtype=torch.float64, device=dev, requires_grad=True)
    out = tb.step(*xs, w, 1200.0, suppress=False)
    gen = torch.Generator(device=dev).manual_seed(7)
    cot = [torch.randn(t.shape, dtype=torch.float64, device=dev, generator=gen)
           / t.detach().abs().max().clamp_min(1e-30) for t in out]
    grads = torch.autograd.grad(out, xs + [w], cot)
    torch.cuda.synchronize()
    L = lib()
    c4, c5 = cot[4].cpu().numpy(), cot[5].cpu().numpy()
    seeds = [c.contiguous() for c in cot[:4]]
    _check(L.oqg_adj_set(g.h, *[_ptr(x) for x in seeds], _dp(c4), _dp(c5)), "adj_set")
    run = AdjointRun(g, every=1)
    _check(L.oqg_pq_save(g.h, _ptr(run.slots[0])), "pq_save")
    _check(L.oqg_adj_step(g.h, _ptr(run.slots[0]), ctypes.c_double(1200.0), ctypes.c_longlong(3)), "adj_step")
    res = [torch.empty(b.shape3, dtype=torch.float64, device=dev) for _ in range(4)]
    lw = torch.empty(b.shape2, dtype=torch.float64, device=dev)
    l1, l2 = np.empty(b.nl - 1), np.empty(b.nl - 1)
    _check(L.oqg_adj_get(g.h, *[_ptr(r) for r in res], _dp(l1), _dp(l2), _ptr(lw)), "adj_get")
    mine = res + [torch.tensor(l1, device=dev), torch.tensor(l2, device=dev), lw]
    for name, a, r in zip(["p", "pm", "q", "qm", "dpi", "dpip", "wekp"], mine, grads):
        err = float((a - r).norm() / r.norm())
        assert err <= 1e-9, "lambda_%s: rel L2 %.3e" % (name, err)
    g.close()


def test_gradient_differentiable_configuration():
    """The differentiable configuration itself: 3-layer ocean at 257x257,
    dx 20 km, 200 leapfrog steps, J = ekei(1) of the final state, checkpoint
    every 20 steps; gradients with respect to the initial psi (FP64) and the
    wind-stress curl field (FP32) against central differences (eps 1e-4
    relative) along 16 seeded random directions."""
    b = ocean_double_gyre(257, dx=20.0e3)
    g = QG(b)
    n, every = 200, 20
    psi0 = torch.tensor(initial_psi(b, seed=11), dtype=torch.float64, device="cuda")
    curl0 = torch.tensor(b.fnot * _forcing(b), dtype=torch.float32, device="cuda")

    def J(psi, curl):
        with torch.no_grad():
            return float(_objective(b, QGRun.apply(psi, curl, g, n, TDT, every)))

    psi = psi0.clone().requires_grad_(True)
    curl = curl0.clone().requires_grad_(True)
    _objective(b, QGRun.apply(psi, curl, g, n, TDT, every)).backward()
    gpsi, gcurl = psi.grad.double(), curl.grad.double()
    gen = torch.Generator(device="cuda").manual_seed(2024)
    worst = 0.0
    for d in range(16):
        dp = torch.randn(b.shape3, dtype=torch.float64, device="cuda", generator=gen)
        dp[:, [0, -1], :] = 0.0
        dp[:, :, [0, -1]] = 0.0
        dc = torch.randn(b.shape2, dtype=torch.float64, device="cuda", generator=gen)
        eps_p = 1e-4 * float(psi0.norm()) / float(dp.norm())
        eps_c = 1e-4 * float(curl0.double().norm()) / float(dc.norm())
        cp = (curl0.double() + eps_c * dc).float()
        cm = (curl0.double() - eps_c * dc).float()
        fd = (J(psi0 + eps_p * dp, cp) - J(psi0 - eps_p * dp, cm)) / 2.0
        # the FP32 control moves by what FP32 represents of the step
        dcp = (cp.double() - cm.double()) / 2.0
        an = eps_p * float((gpsi * dp).sum()) + float((gcurl * dcp).sum())
        worst = max(worst, abs(fd - an) / abs(an))
        assert abs(fd - an) <= 1e-6 * abs(an), "direction %d: fd %.12e adjoint %.12e" % (d, fd, an)
    g.close()
