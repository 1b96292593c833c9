"""TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.

ctypes wrapper of the CPU FP64 oracle (oracle/oqg_oracle.cpp), a restatement
of OpenQG's per-timestep QG core (src/qg/core.F90:16-33 and the routines it
calls).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
use it, always as the checker or the timed CPU baseline, never as the thing
measured on the GPU.

Parity pins: the reference's Helmholtz residual tests
(src/tests/test_inhomog.F90:123-154, 208-240), the mode-matrix identity check
(src/qg/modes.F90:148-161), an O(n^2) long-double DST, Arakawa-Jacobian
conservation and mass-constraint closure.  The reference has no golden
vectors for the step itself; bitwise FFTW/LAPACK parity is unpinned.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from openqg_b200.params import Basin, QgMonitor

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "build", "liboqg_oracle.so")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, OpenMP)."""
    if force or not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(
            os.path.join(_HERE, "oqg_oracle.cpp")):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_void_p]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_last_error.restype = ctypes.c_char_p
        for name, nargs in [("orc_set_state", 2), ("orc_get_state", 4),
                            ("orc_get_constraints", 6), ("orc_get_modes", 4),
                            ("orc_get_homog", 2), ("orc_jacobian", 3)]:
            f = getattr(L, name)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_void_p] + [_dp] * nargs
        L.orc_set_state_full.restype = ctypes.c_int
        L.orc_set_state_full.argtypes = [ctypes.c_void_p] + [_dp] * 10
        L.orc_set_forcing.restype = ctypes.c_int
        L.orc_set_forcing.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_double, ctypes.c_double]
        L.orc_step.restype = ctypes.c_int
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.orc_set_step_index.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
        L.orc_suppress.argtypes = [ctypes.c_void_p]
        L.orc_diag.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp]
        L.orc_diagno.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_double, ctypes.c_double,
                                 ctypes.POINTER(QgMonitor)]
        L.orc_solve_inhomog.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_generate_homog_soln.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_set_rdm2.argtypes = [ctypes.c_void_p, _dp]
        L.orc_del2.argtypes = [ctypes.c_void_p, _dp, ctypes.c_double, _dp]
        L.orc_int_P_dA.restype = ctypes.c_double
        L.orc_int_P_dA.argtypes = [ctypes.c_void_p, _dp]
        L.orc_dst1.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_dst1_direct_ld.argtypes = [ctypes.c_int, _dp, _dp]
        L.orc_rfft.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_irfft.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_ekman_from_tau.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _dp]
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


class Oracle:
    """One basin of the CPU restatement.  Arrays are (nl, nyp, nxp) C-order,
    i.e. Fortran (nxp, nyp, nl)."""

    def __init__(self, basin: Basin):
        self.b = basin
        self._prm = basin.to_c()
        self.h = lib().orc_create(ctypes.byref(self._prm))
        if not self.h:
            raise RuntimeError("oracle create failed: %s" % lib().orc_last_error().decode())

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # state -------------------------------------------------------------
    def set_state(self, p, pm):
        p = np.ascontiguousarray(p, dtype=np.float64)
        pm = np.ascontiguousarray(pm, dtype=np.float64)
        lib().orc_set_state(self.h, _p(p), _p(pm))

    def set_state_full(self, p, pm, q, qm, dpi, dpip, cs=None, cn=None, csp=None, cnp=None):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
                for a in (p, pm, q, qm, dpi, dpip, cs, cn, csp, cnp)]
        lib().orc_set_state_full(self.h, *[_p(a) for a in arrs])

    def get_state(self):
        sh = self.b.shape3
        p, pm, q, qm = (np.empty(sh) for _ in range(4))
        lib().orc_get_state(self.h, _p(p), _p(pm), _p(q), _p(qm))
        return p, pm, q, qm

    def get_constraints(self):
        nl = self.b.nl
        dpi, dpip = np.empty(nl - 1), np.empty(nl - 1)
        cs, cn, csp, cnp = (np.empty(nl) for _ in range(4))
        lib().orc_get_constraints(self.h, _p(dpi), _p(dpip), _p(cs), _p(cn), _p(csp), _p(cnp))
        return dict(dpi=dpi, dpip=dpip, cs=cs, cn=cn, csp=csp, cnp=cnp)

    def set_forcing(self, wekp=None, ent=None, txis=0.0, txin=0.0):
        w = np.ascontiguousarray(wekp, dtype=np.float64) if wekp is not None else None
        e = np.ascontiguousarray(ent, dtype=np.float64) if ent is not None else None
        lib().orc_set_forcing(self.h, _p(w), _p(e), txis, txin)

    def step(self, tdt, nsteps=1):
        lib().orc_step(self.h, tdt, nsteps)

    def set_step_index(self, nt):
        lib().orc_set_step_index(self.h, nt)

    def suppress(self):
        lib().orc_suppress(self.h)

    def diag(self):
        nl = self.b.nl
        e, smin, smax, c = (np.empty(nl) for _ in range(4))
        lib().orc_diag(self.h, _p(e), _p(smin), _p(smax), _p(c))
        return dict(ekei=e, sfmin=smin, sfmax=smax, circ=c)

    def diagno(self, taux=None, tauy=None, tsec=0.0, tdt=0.0, mon=None):
        """qg_diagno (qg_monitor.F90:219-383); mon carries state between calls."""
        mon = mon if mon is not None else QgMonitor()
        tx = None if taux is None else np.ascontiguousarray(taux, dtype=np.float64)
        ty = None if tauy is None else np.ascontiguousarray(tauy, dtype=np.float64)
        lib().orc_diagno(self.h, _p(tx), _p(ty), float(tsec), float(tdt), ctypes.byref(mon))
        return mon.as_dict(self.b.nl), mon

    # pieces of the path ---------------------------------------------------
    def solve_inhomog(self, m, rhs):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        out = np.empty(self.b.shape2)
        lib().orc_solve_inhomog(self.h, m, _p(rhs), _p(out))
        return out

    def generate_homog_soln(self, m, L):
        L = np.ascontiguousarray(L, dtype=np.float64)
        out = np.empty(self.b.shape2)
        lib().orc_generate_homog_soln(self.h, m, _p(L), _p(out))
        return out

    def modes(self):
        nl = self.b.nl
        amat, ctl2m, ctm2l = (np.empty(nl * nl) for _ in range(3))
        rdm2 = np.empty(nl)
        lib().orc_get_modes(self.h, _p(amat), _p(rdm2), _p(ctl2m), _p(ctm2l))
        f = lambda a: a.reshape(nl, nl).T.copy()   # column-major -> [row, col]
        return dict(amat=f(amat), rdm2=rdm2, ctl2m=f(ctl2m), ctm2l=f(ctm2l))

    def homog(self):
        b = self.b
        if b.cyclic:
            a = np.empty((b.nl, b.nyp)); c = np.empty((b.nl, b.nyp))
            lib().orc_get_homog(self.h, _p(a), _p(c))
            return a, c
        a = np.empty((b.nl - 1, b.nyp, b.nxp))
        lib().orc_get_homog(self.h, _p(a), None)
        return a

    def set_rdm2(self, rdm2):
        r = np.ascontiguousarray(rdm2, dtype=np.float64)
        lib().orc_set_rdm2(self.h, _p(r))

    def jacobian(self, p2, q2):
        p2 = np.ascontiguousarray(p2, dtype=np.float64)
        q2 = np.ascontiguousarray(q2, dtype=np.float64)
        out = np.empty(self.b.shape2)
        lib().orc_jacobian(self.h, _p(p2), _p(q2), _p(out))
        return out

    def del2(self, f2, alpha):
        f2 = np.ascontiguousarray(f2, dtype=np.float64)
        out = np.empty(self.b.shape2)
        lib().orc_del2(self.h, _p(f2), alpha, _p(out))
        return out

    def int_P_dA(self, f2):
        f2 = np.ascontiguousarray(f2, dtype=np.float64)
        return lib().orc_int_P_dA(self.h, _p(f2))


def dst1(x: np.ndarray) -> np.ndarray:
    """FFTW RODFT00 along the last axis (oracle FFT)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[-1]
    rows = x.size // n
    out = np.empty_like(x)
    lib().orc_dst1(n, rows, _p(x), _p(out))
    return out


def dst1_direct(x: np.ndarray) -> np.ndarray:
    """O(n^2) long-double DST-I of a 1-D vector."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    lib().orc_dst1_direct_ld(x.size, _p(x), _p(out))
    return out


def rfft(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    N = x.shape[-1]
    rows = x.size // N
    out = np.empty(x.shape[:-1] + (N // 2 + 1,), dtype=np.complex128)
    lib().orc_rfft(N, rows, _p(x), out.ctypes.data_as(_dp))
    return out


def irfft(X: np.ndarray, N: int) -> np.ndarray:
    X = np.ascontiguousarray(X, dtype=np.complex128)
    rows = X.size // (N // 2 + 1)
    out = np.empty(X.shape[:-1] + (N,))
    lib().orc_irfft(N, rows, X.ctypes.data_as(_dp), _p(out))
    return out


def ekman_from_tau(basin: Basin, taux, tauy):
    """ekman_from_tau (src/coupler/ekman.F90:53-83): (wekp, txis, txin)."""
    prm = basin.to_c()
    taux = np.ascontiguousarray(taux, dtype=np.float64)
    tauy = np.ascontiguousarray(tauy, dtype=np.float64)
    w = np.empty(basin.shape2)
    ts, tn = ctypes.c_double(0), ctypes.c_double(0)
    lib().orc_ekman_from_tau(ctypes.byref(prm), _p(taux), _p(tauy), _p(w),
                             ctypes.cast(ctypes.byref(ts), _dp), ctypes.cast(ctypes.byref(tn), _dp))
    return w, ts.value, tn.value
