"""Vectorised numpy restatements of a few reference stencils (test helpers).

Used to cross-check the C++ oracle and the GPU kernels against a second,
independent reading of src/glam/numerics.F90 and src/qg/vorsubs.F90.
Arrays are (nyp, nxp) or (nl, nyp, nxp) C-order, i.e. Fortran (nxp, nyp[, nl]).
"""
import numpy as np


def dP2dx2_bc(p, dx, alpha, cyclic):
    """numerics.F90:427-448."""
    fac = 1.0 / (dx * dx)
    o = np.zeros_like(p)
    o[..., :, 1:-1] = fac * (p[..., :, :-2] + p[..., :, 2:] - 2.0 * p[..., :, 1:-1])
    if not cyclic:
        c = fac * alpha / (0.5 * alpha + 1.0)
        o[..., :, 0] = c * (p[..., :, 1] - p[..., :, 0])
        o[..., :, -1] = -c * (p[..., :, -1] - p[..., :, -2])
    else:
        o[..., :, 0] = fac * (p[..., :, -2] + p[..., :, 1] - 2.0 * p[..., :, 0])
        o[..., :, -1] = o[..., :, 0]
    o[..., 0, :] = 0.0
    o[..., -1, :] = 0.0
    return o


def dP2dy2_bc(p, dy, alpha, cyclic):
    """numerics.F90:450-468."""
    fac = 1.0 / (dy * dy)
    o = np.zeros_like(p)
    o[..., 1:-1, :] = fac * (p[..., :-2, :] + p[..., 2:, :] - 2.0 * p[..., 1:-1, :])
    c = fac * alpha / (0.5 * alpha + 1.0)
    o[..., 0, :] = c * (p[..., 1, :] - p[..., 0, :])
    o[..., -1, :] = -c * (p[..., -1, :] - p[..., -2, :])
    if not cyclic:
        o[..., :, 0] = 0.0
        o[..., :, -1] = 0.0
    return o


def del2_bc(p, dx, dy, alpha, cyclic):
    """del2_P_bc, numerics.F90:410-425."""
    return dP2dx2_bc(p, dx, alpha, cyclic) + dP2dy2_bc(p, dy, alpha, cyclic)


def qcomp(p, amat, basin):
    """qcomp, vorsubs.F90:27-56 (p is (nl, nyp, nxp))."""
    b = basin
    q = del2_bc(p, b.dx, b.dy, b.bcco, b.cyclic) / b.fnot
    kt = b.ktopo() - 1
    if b.ddyn is not None:
        q[kt] += np.asarray(b.ddyn).reshape(b.nyp, b.nxp)
    q += b.beta * b.yprel[None, :, None]
    q -= b.fnot * np.einsum("kl,lji->kji", amat, p)
    return q


def dPdx_2(f, cyclic):
    o = np.zeros_like(f)
    o[..., :, 1:-1] = f[..., :, 2:] - f[..., :, :-2]
    if cyclic:
        o[..., :, 0] = f[..., :, 1] - f[..., :, -2]
    o[..., :, -1] = o[..., :, 0]
    return o


def dPdy_2(f):
    o = np.zeros_like(f)
    o[..., 1:-1, :] = f[..., 2:, :] - f[..., :-2, :]
    return o


def jacobian(p, q, dx, dy, f0, cyclic):
    """jacobian, numerics.F90:340-373."""
    fac = 1.0 / (3.0 * (2.0 * dx) * (2.0 * dy) * f0)
    px, py, qx, qy = dPdx_2(p, cyclic), dPdy_2(p), dPdx_2(q, cyclic), dPdy_2(q)
    return fac * (qx * py - qy * px + dPdx_2(q * py, cyclic) - dPdy_2(q * px)
                  + dPdy_2(p * qx) - dPdx_2(p * qy, cyclic))


def int_P_dA(f, dx, dy):
    """Trapezoid area integral, numerics.F90:188-204."""
    w = np.ones(f.shape[-2:])
    w[0, :] *= 0.5
    w[-1, :] *= 0.5
    w[:, 0] *= 0.5
    w[:, -1] *= 0.5
    return (f * w).sum(axis=(-2, -1)) * dx * dy


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
