"""The plain-PyTorch restatement of the closed-box step (oracle/torch_step.py),
the autograd reference of the adjoint, pinned against the C++ oracle: states
within 1e-13 relative L2 over three steps (the first followed by
suppress_comp_mode), and set_state's q, qm and mass constraints."""
import numpy as np
import pytest
import torch

import oracle
from oracle.torch_step import TorchBox
from openqg_b200.params import double_gyre_tau, initial_psi, ocean_double_gyre
from tests.qg_numpy import rel_l2


def _setup(n=33, seed=1, nl=3):
    b = ocean_double_gyre(n, dx=40.0e3, ah4=2.0e11)
    b.ah2 = [300.0, 200.0, 100.0]
    if nl == 2:
        b.h, b.gp, b.ah2, b.ah4 = [1000.0, 3000.0], [0.02], [300.0, 100.0], [2.0e11] * 2
    elif nl == 4:
        b.h, b.gp = [300.0, 500.0, 800.0, 2400.0], [0.04, 0.02, 0.01]
        b.ah2, b.ah4 = [300.0, 200.0, 150.0, 100.0], [2.0e11] * 4
    o = oracle.Oracle(b)
    p = b.fnot * initial_psi(b, seed=seed)
    pm = p + 0.05 * b.fnot * initial_psi(b, seed=seed + 5)
    tx, ty = double_gyre_tau(b)
    w, ts, tn = oracle.ekman_from_tau(b, tx, ty)
    o.set_state(p, pm)
    o.set_forcing(w, None, ts, tn)
    return b, o, p, pm, w.reshape(b.shape2)


def test_init_state_matches_oracle():
    b, o, p, pm, _ = _setup()
    tb = TorchBox(b, o)
    st = tb.init_state(torch.tensor(p), torch.tensor(pm))
    ref = o.get_state()
    for a, r in zip(st[:4], ref):
        assert rel_l2(a.numpy(), r) <= 1e-14
    c = o.get_constraints()
    assert rel_l2(st[4].numpy(), c["dpi"]) <= 1e-13
    assert rel_l2(st[5].numpy(), c["dpip"]) <= 1e-13


@pytest.mark.parametrize("nl", [2, 3, 4])
def test_steps_match_oracle(nl):
    b, o, p, pm, w = _setup(nl=nl)
    tb = TorchBox(b, o)
    st = tb.init_state(torch.tensor(p), torch.tensor(pm))
    W = torch.tensor(w)
    for s in range(1, 4):
        st = tb.step(*st, W, 3600.0, suppress=(s - 1) % b.suppress_period == 0)
        o.step(3600.0, 1)
        for a, r in zip(st[:4], o.get_state()):
            assert rel_l2(a.numpy(), r) <= 1e-13
        c = o.get_constraints()
        assert rel_l2(st[4].numpy(), c["dpi"]) <= 1e-13


def test_step_is_differentiable():
    """autograd runs through the restated step and agrees with a central
    difference of it (the restatement's own sanity, eps 1e-6 relative)."""
    b, o, p, pm, w = _setup(n=17)
    tb = TorchBox(b, o)
    x = torch.tensor(p, requires_grad=True)
    st = tb.init_state(x, x)
    out = tb.step(*st, torch.tensor(w), 3600.0)
    J = (out[0] ** 2).sum()
    (g,) = torch.autograd.grad(J, [x])
    rng = np.random.default_rng(0)
    d = torch.tensor(rng.standard_normal(p.shape))
    eps = 1e-6 * float(x.detach().norm()) / float(d.norm())

    def f(y):
        s = tb.init_state(y, y)
        return float((tb.step(*s, torch.tensor(w), 3600.0)[0] ** 2).sum())

    with torch.no_grad():
        fd = (f(x + eps * d) - f(x - eps * d)) / (2 * eps)
    an = float((g * d).sum())
    assert abs(fd - an) <= 1e-6 * abs(an)
