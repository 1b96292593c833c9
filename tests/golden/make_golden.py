"""Writes the golden step fixtures of this directory from the FP64 oracle.

The reference's own tests pin the Helmholtz solver and the mode matrices by
residuals, not by stored vectors, and the Fortran step cannot be built here;
these fixtures freeze the oracle's step on seeded inputs so that both the
oracle (CPU tests) and the CUDA path (GPU tests) are checked against the
same committed numbers.

    python tests/golden/make_golden.py      # rewrites golden_*.npz
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from openqg_b200.params import atmos_channel, double_gyre_tau, initial_psi, ocean_double_gyre  # noqa: E402


def channel_tau(b, amp=0.1):
    yl = (b.nyp - 1) * b.dy
    y = np.arange(b.nyp) * b.dy
    taux = np.repeat((amp * np.sin(np.pi * y / yl))[:, None], b.nxp, axis=1)
    return taux, np.zeros_like(taux)


def entrainment(b, seed, amp=1e-6):
    rng = np.random.default_rng(seed)
    yy, xx = np.meshgrid(np.linspace(0, 1, b.nyp), np.linspace(0, 1, b.nxp), indexing="ij")
    e = np.zeros((b.nl - 1,) + b.shape2)
    for k in range(b.nl - 1):
        e[k] = amp * (np.sin(2 * np.pi * xx * (k + 1)) * np.cos(np.pi * yy) + 0.3 * rng.standard_normal(b.shape2))
        if b.cyclic:
            e[k][:, -1] = e[k][:, 0]
    return e


# name -> (basin, tdt, psi amplitude, with entrainment)
CASES = {
    "box33": (lambda: ocean_double_gyre(33), 3600.0, 1.0, False),
    "box33ent": (lambda: ocean_double_gyre(33), 3600.0, 1.0, True),
    "chan49x25": (lambda: atmos_channel(49, 25), 360.0, 30.0, True),
}


def inputs(name):
    mk, tdt, amp, with_ent = CASES[name]
    b = mk()
    p = b.fnot * initial_psi(b, 3) * amp
    pm = 0.5 * p + 0.5 * b.fnot * initial_psi(b, 10) * amp * 0.5
    taux, tauy = channel_tau(b) if b.cyclic else double_gyre_tau(b)
    wekp, txis, txin = oracle.ekman_from_tau(b, taux, tauy)
    ent = entrainment(b, 4) if with_ent else None
    return b, tdt, p, pm, wekp, ent, txis, txin


def run(name):
    b, tdt, p, pm, wekp, ent, txis, txin = inputs(name)
    o = oracle.Oracle(b)
    o.set_state(p, pm)
    o.set_forcing(wekp, ent, txis, txin)
    o.step(tdt, 1)
    p1, _, q1, _ = o.get_state()
    o.step(tdt, 9)
    p10, _, q10, _ = o.get_state()
    c = o.get_constraints()
    out = dict(p0=p, pm0=pm, wekp=wekp, txis=txis, txin=txin, tdt=tdt,
               p1=p1, q1=q1, p10=p10, q10=q10, dpi10=c["dpi"])
    if ent is not None:
        out["ent"] = ent
    return out


def main():
    for name in CASES:
        path = os.path.join(HERE, "golden_%s.npz" % name)
        np.savez_compressed(path, **run(name))
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
