"""Host-side mirror of OpenQG's QG-core interface over the C ABI (include/oqg.h).

The names follow the reference so a caller reads the same program:

    qg = init_qg(basin)                     # qg.F90:60-103   init_qg
    qg.set_state(p, pm)                     # init_pv + init_constraint + init_mass_constr
    step_qg(tdt, ent, wekp, txis, txin, qg) # core.F90:16-33  one step
    suppress_comp_mode(qg)                  # driver.F90:174-189

Arrays are numpy FP64 with shape (nl, nyp, nxp) in C order, which is the
memory layout of the reference's Fortran (nxp, nyp, nl) arrays.  Every call
runs on the GPU through liboqg.so; there is no CPU fallback, and a missing
library or device raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from .params import Basin, OqgAmlParams, OqgOmlParams, OqgRadCoeffs, QgMonitor, STATUS

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboqg.so")
_dp = ctypes.POINTER(ctypes.c_double)
_lib = None


class OqgError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__("%s failed: %s (%s)" % (where, STATUS.get(code, code), msg))
        self.code = code


def lib():
    """Loads liboqg.so (built by openqg_b200.build); raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("liboqg.so is not built; run `python -m openqg_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    L.oqg_last_error.restype = ctypes.c_char_p
    L.oqg_version.argtypes = [ctypes.c_char_p, ctypes.c_int]
    L.oqg_create.argtypes = [vp, ctypes.POINTER(vp)]
    L.oqg_destroy.argtypes = [vp]
    L.oqg_set_state.argtypes = [vp, _dp, _dp]
    L.oqg_set_state_full.argtypes = [vp] + [_dp] * 10
    L.oqg_get_state.argtypes = [vp, _dp, _dp, _dp, _dp]
    L.oqg_get_p_layer.argtypes = [vp, ctypes.c_int, _dp]
    L.oqg_get_constraints.argtypes = [vp] + [_dp] * 6
    L.oqg_set_forcing.argtypes = [vp, _dp, _dp, ctypes.c_double, ctypes.c_double]
    L.oqg_step.argtypes = [vp, ctypes.c_double, ctypes.c_int]
    L.oqg_set_step_index.argtypes = [vp, ctypes.c_longlong]
    L.oqg_get_step_index.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.oqg_suppress.argtypes = [vp]
    L.oqg_sync.argtypes = [vp]
    L.oqg_set_wait_limit.argtypes = [vp, ctypes.c_longlong]
    L.oqg_check_finite.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.oqg_diag.argtypes = [vp, _dp, _dp, _dp, _dp]
    L.oqg_diag_noalloc.argtypes = [vp, _dp, _dp, _dp, _dp]
    L.oqg_valids.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, _dp,
                             ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int)]
    L.oqg_diagno.argtypes = [vp, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.POINTER(QgMonitor)]
    L.oqg_solve_inhomog.argtypes = [vp, ctypes.c_int, _dp, _dp]
    L.oqg_int_P_dA.argtypes = [vp, _dp, _dp]
    L.oqg_generate_homog_soln.argtypes = [vp, ctypes.c_int, _dp, _dp]
    L.oqg_get_modes.argtypes = [vp, _dp, _dp, _dp, _dp]
    L.oqg_ekman_from_tau.argtypes = [vp, _dp, _dp, _dp, _dp, _dp]
    L.oqg_device_state.argtypes = [vp] + [ctypes.POINTER(vp)] * 4 + [ctypes.POINTER(ctypes.c_int)] * 2
    L.oqg_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.oqg_step_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.oqg_launch_floor.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.oqg_profile_phases.argtypes = [vp, ctypes.c_double, ctypes.c_int, _dp]
    L.oqg_ensemble_create.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp)]
    L.oqg_ensemble_destroy.argtypes = [vp]
    L.oqg_ensemble_set_state.argtypes = [vp, ctypes.c_int, _dp, _dp]
    L.oqg_ensemble_get_state.argtypes = [vp, ctypes.c_int, _dp, _dp, _dp, _dp]
    L.oqg_ensemble_set_forcing.argtypes = [vp, ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_double]
    L.oqg_ensemble_step.argtypes = [vp, _dp, ctypes.c_int]
    L.oqg_ensemble_sync.argtypes = [vp]
    L.oqg_ensemble_stream.argtypes = [vp, ctypes.POINTER(vp)]
    L.oqg_state_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
    L.oqg_state_save.argtypes = [vp, vp]
    L.oqg_state_load.argtypes = [vp, vp]
    L.oqg_pq_save.argtypes = [vp, vp]
    L.oqg_adj_set.argtypes = [vp, vp, vp, vp, vp, _dp, _dp]
    L.oqg_adj_get.argtypes = [vp, vp, vp, vp, vp, _dp, _dp, vp]
    L.oqg_adj_step.argtypes = [vp, vp, ctypes.c_double, ctypes.c_longlong]
    L.oqg_adj_initial.argtypes = [vp, vp, vp]
    L.oqg_oml_create.argtypes = [vp, ctypes.POINTER(OqgOmlParams), ctypes.POINTER(vp)]
    L.oqg_oml_destroy.argtypes = [vp]
    L.oqg_oml_set_sst.argtypes = [vp, vp, vp]
    L.oqg_oml_get_sst.argtypes = [vp, vp, vp]
    L.oqg_ocean_forcing.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.c_double]
    L.oqg_get_forcing.argtypes = [vp, _dp, _dp]
    L.oqg_oml_couple.argtypes = [vp, vp, ctypes.c_double]
    L.oqg_xforc.argtypes = [vp, vp]
    L.oqg_oml_tau_udiff.argtypes = [vp, ctypes.c_int]
    L.oqg_compute_forcing.argtypes = [vp, ctypes.POINTER(OqgRadCoeffs)]
    L.oqg_get_fluxes.argtypes = [vp, vp, vp]
    L.oqg_aml_create.argtypes = [vp, ctypes.POINTER(OqgAmlParams), vp, vp, ctypes.POINTER(vp)]
    L.oqg_aml_destroy.argtypes = [vp]
    L.oqg_aml_set_state.argtypes = [vp, vp, vp, vp, vp]
    L.oqg_aml_get_state.argtypes = [vp, vp, vp, vp, vp]
    L.oqg_atmos_forcing.argtypes = [vp, vp, vp, vp, ctypes.c_int, ctypes.c_double]
    L.oqg_ensemble_autotune.argtypes = [vp, _dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _dp]
    L.oqg_autotune.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _dp]
    L.oqg_get_vty.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.oqg_autotune_ysolve.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_double)]
    L.oqg_get_ysolve_warps.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.oqg_set_vty.argtypes = [vp, ctypes.c_int]
    L.oqg_set_ysolve_warps.argtypes = [vp, ctypes.c_int]
    L.oqg_set_xinv_sep.argtypes = [vp, ctypes.c_int]
    L.oqg_get_xinv_sep.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.oqg_autotune_xinv.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_double)]
    L.oqg_adj_segment.argtypes = [vp, vp, vp, ctypes.c_size_t, ctypes.c_int, ctypes.c_double, ctypes.c_longlong]
    _lib = L
    return L


def _check(rc: int, where: str):
    if rc != 0:
        raise OqgError(rc, where, lib().oqg_last_error().decode())


def _p(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _f64(a, shape=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.size != int(np.prod(shape)):
        raise ValueError("expected %s values, got %d" % (shape, a.size))
    return a


def version() -> str:
    buf = ctypes.create_string_buffer(256)
    lib().oqg_version(buf, 256)
    return buf.value.decode()


class QG:
    """Device-resident qg_type (qg.F90:17-53) of one basin."""

    def __init__(self, basin: Basin):
        self.b = basin
        self._prm = basin.to_c()
        h = ctypes.c_void_p()
        _check(lib().oqg_create(ctypes.byref(self._prm), ctypes.byref(h)), "oqg_create")
        self.h = h

    # lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            lib().oqg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # state ----------------------------------------------------------------
    def set_state(self, p, pm):
        """Restart semantics: q, qm and constraints recomputed from p, pm."""
        p = _f64(p, self.b.shape3)
        pm = _f64(pm, self.b.shape3)
        _check(lib().oqg_set_state(self.h, _p(p), _p(pm)), "oqg_set_state")

    def set_state_full(self, p, pm, q, qm, dpi, dpip, cs=None, cn=None, csp=None, cnp=None):
        arrs = [_f64(a) for a in (p, pm, q, qm, dpi, dpip, cs, cn, csp, cnp)]
        _check(lib().oqg_set_state_full(self.h, *[_p(a) for a in arrs]), "oqg_set_state_full")

    def get_state(self):
        sh = self.b.shape3
        p, pm, q, qm = (np.empty(sh) for _ in range(4))
        _check(lib().oqg_get_state(self.h, _p(p), _p(pm), _p(q), _p(qm)), "oqg_get_state")
        return p, pm, q, qm

    @property
    def p(self):
        out = np.empty(self.b.shape3)
        _check(lib().oqg_get_state(self.h, _p(out), None, None, None), "oqg_get_state")
        return out

    def p_layer(self, k: int = 0, out: Optional[np.ndarray] = None):
        if out is None:
            out = np.empty(self.b.shape2)
        _check(lib().oqg_get_p_layer(self.h, k, _p(out)), "oqg_get_p_layer")
        return out

    def constraints(self):
        nl = self.b.nl
        dpi, dpip = np.empty(nl - 1), np.empty(nl - 1)
        cs, cn, csp, cnp = (np.empty(nl) for _ in range(4))
        _check(lib().oqg_get_constraints(self.h, _p(dpi), _p(dpip), _p(cs), _p(cn), _p(csp), _p(cnp)),
               "oqg_get_constraints")
        return dict(dpi=dpi, dpip=dpip, cs=cs, cn=cn, csp=csp, cnp=cnp)

    # forcing and stepping ------------------------------------------------------
    def set_forcing(self, wekp=None, ent=None, txis=0.0, txin=0.0):
        w = _f64(wekp, self.b.shape2)
        e = _f64(ent, (self.b.nl - 1,) + self.b.shape2)
        _check(lib().oqg_set_forcing(self.h, _p(w), _p(e), float(txis), float(txin)), "oqg_set_forcing")

    def step(self, tdt: float, nsteps: int = 1):
        _check(lib().oqg_step(self.h, float(tdt), int(nsteps)), "oqg_step")

    def set_step_index(self, steps_done: int):
        _check(lib().oqg_set_step_index(self.h, int(steps_done)), "oqg_set_step_index")

    def step_index(self) -> int:
        v = ctypes.c_longlong()
        _check(lib().oqg_get_step_index(self.h, ctypes.byref(v)), "oqg_get_step_index")
        return v.value

    def suppress(self):
        _check(lib().oqg_suppress(self.h), "oqg_suppress")

    def sync(self):
        _check(lib().oqg_sync(self.h), "oqg_sync")

    def check_finite(self) -> int:
        v = ctypes.c_longlong()
        rc = lib().oqg_check_finite(self.h, ctypes.byref(v))
        if rc not in (0, 3):
            _check(rc, "oqg_check_finite")
        return v.value

    def diag(self):
        nl = self.b.nl
        e, smin, smax, c = (np.empty(nl) for _ in range(4))
        _check(lib().oqg_diag(self.h, _p(e), _p(smin), _p(smax), _p(c)), "oqg_diag")
        return dict(ekei=e, sfmin=smin, sfmax=smax, circ=c)

    def diagno(self, taux=None, tauy=None, tsec=0.0, tdt=0.0, mon: Optional[QgMonitor] = None):
        """qg_diagno (qg_monitor.F90:219-383) on the device.  mon carries the
        time-rate state between calls; returns (dict of the record, mon)."""
        mon = mon if mon is not None else QgMonitor()
        tx = _f64(taux, self.b.shape2)
        ty = _f64(tauy, self.b.shape2)
        _check(lib().oqg_diagno(self.h, _p(tx), _p(ty), float(tsec), float(tdt), ctypes.byref(mon)), "oqg_diagno")
        return mon.as_dict(self.b.nl), mon

    def valids(self, pext: float, qext: float, wext: float):
        """valids (valsubs.F90:46-139) for p, q and wekp: (ok, extremes dict,
        count of non-finite values)."""
        ext = np.empty(6)
        bad = ctypes.c_longlong()
        ok = ctypes.c_int()
        _check(lib().oqg_valids(self.h, float(pext), float(qext), float(wext), _p(ext), ctypes.byref(bad),
                                ctypes.byref(ok)), "oqg_valids")
        names = ("pmin", "pmax", "qmin", "qmax", "wmin", "wmax")
        return bool(ok.value), dict(zip(names, ext)), bad.value

    def diag_noalloc(self):
        """diag() through oqg_diag_noalloc: scratch in the library's fixed
        device array, no allocation; it reports failures by status only."""
        nl = self.b.nl
        e, smin, smax, c = (np.empty(nl) for _ in range(4))
        rc = lib().oqg_diag_noalloc(self.h, _p(e), _p(smin), _p(smax), _p(c))
        if rc != 0:
            raise OqgError(rc, "oqg_diag_noalloc", "status only")
        return dict(ekei=e, sfmin=smin, sfmax=smax, circ=c)

    # pieces of the path -----------------------------------------------------------
    def solve_inhomog_eqn(self, m: int, rhs):
        """solve_inhomog_eqn (inhomog.F90:156-168) for mode m (1-based)."""
        rhs = _f64(rhs, self.b.shape2)
        out = np.empty(self.b.shape2)
        _check(lib().oqg_solve_inhomog(self.h, int(m), _p(rhs), _p(out)), "oqg_solve_inhomog")
        return out

    def int_P_dA(self, f) -> float:
        """int_P_dA (numerics.F90:165-204) of a (nyp, nxp) field, on the
        device with compensated summation."""
        f = _f64(f, self.b.shape2)
        out = np.empty(1)
        _check(lib().oqg_int_P_dA(self.h, _p(f), _p(out)), "oqg_int_P_dA")
        return float(out[0])

    def generate_homog_soln(self, m: int, L):
        L = _f64(L, self.b.shape2)
        out = np.empty(self.b.shape2)
        _check(lib().oqg_generate_homog_soln(self.h, int(m), _p(L), _p(out)), "oqg_generate_homog_soln")
        return out

    def modes(self):
        nl = self.b.nl
        amat, ctl2m, ctm2l = (np.empty(nl * nl) for _ in range(3))
        rdm2 = np.empty(nl)
        _check(lib().oqg_get_modes(self.h, _p(amat), _p(rdm2), _p(ctl2m), _p(ctm2l)), "oqg_get_modes")
        f = lambda a: a.reshape(nl, nl).T.copy()
        return dict(amat=f(amat), rdm2=rdm2, ctl2m=f(ctl2m), ctm2l=f(ctm2l))

    def device_state(self):
        """(p, pm, q, qm) device pointers, row pitch (elements), element bytes."""
        ptr = [ctypes.c_void_p() for _ in range(4)]
        pitch, eb = ctypes.c_int(), ctypes.c_int()
        _check(lib().oqg_device_state(self.h, *[ctypes.byref(x) for x in ptr],
                                      ctypes.byref(pitch), ctypes.byref(eb)), "oqg_device_state")
        return [x.value for x in ptr], pitch.value, eb.value

    def profile_phases(self, tdt: float, nsteps: int):
        """Mean device ms per launch of the kernels of a step: vorticity,
        forward transform, y-solve, inverse transform, and the assembly when
        it runs as a launch of its own (else 0)."""
        ms = np.zeros(5)
        _check(lib().oqg_profile_phases(self.h, float(tdt), int(nsteps), _p(ms)), "oqg_profile_phases")
        return ms

    def autotune(self, tdt: float, nsteps: int = 20):
        """Measures the vorticity kernel's tile heights on the device and keeps
        the fastest (oqg_autotune); returns (height, {height: ms per step})."""
        best = ctypes.c_int()
        ms = np.full(18, np.nan)
        _check(lib().oqg_autotune(self.h, float(tdt), int(nsteps), ctypes.byref(best), _p(ms)), "oqg_autotune")
        return best.value, {v: float(ms[v]) for v in range(8, 18) if np.isfinite(ms[v])}

    def autotune_ysolve(self, tdt: float, nsteps: int = 20):
        """Measures the y-solve with 1, 2 and 4 warps per column and keeps the
        fastest; returns (warps, {warps: ms per step})."""
        best = ctypes.c_int()
        ms = (ctypes.c_double * 3)()
        _check(lib().oqg_autotune_ysolve(self.h, float(tdt), int(nsteps), ctypes.byref(best), ms),
               "oqg_autotune_ysolve")
        return best.value, {w: ms[i] for i, w in enumerate((1, 2, 4)) if ms[i] >= 0}

    def set_tile_rows(self, rows: int):
        """Fixes the vorticity tile height (8, 12 or 16) without measuring."""
        _check(lib().oqg_set_vty(self.h, int(rows)), "oqg_set_vty")

    def set_ysolve_warps(self, warps: int):
        """Fixes the y-solve's warps per column (1, 2 or 4) without measuring."""
        _check(lib().oqg_set_ysolve_warps(self.h, int(warps)), "oqg_set_ysolve_warps")

    def set_xinv_sep(self, on: bool):
        """The inverse transforms as a launch of their own and a one-pass
        assembly (on), or one kernel for both (off)."""
        _check(lib().oqg_set_xinv_sep(self.h, 1 if on else 0), "oqg_set_xinv_sep")

    def autotune_xinv(self, tdt: float, nsteps: int = 20):
        """Grids below 1025 points: measures the inverse transform and
        assembly as one kernel and as two launches and keeps the faster;
        returns (two_launches, {False: ms, True: ms}) for the forms measured."""
        best = ctypes.c_int()
        ms = (ctypes.c_double * 2)()
        _check(lib().oqg_autotune_xinv(self.h, float(tdt), int(nsteps), ctypes.byref(best), ms),
               "oqg_autotune_xinv")
        return bool(best.value), {bool(i): ms[i] for i in range(2) if ms[i] >= 0}

    def xinv_sep(self) -> bool:
        v = ctypes.c_int()
        _check(lib().oqg_get_xinv_sep(self.h, ctypes.byref(v)), "oqg_get_xinv_sep")
        return bool(v.value)

    def ysolve_warps(self) -> int:
        v = ctypes.c_int()
        _check(lib().oqg_get_ysolve_warps(self.h, ctypes.byref(v)), "oqg_get_ysolve_warps")
        return v.value

    def tile_rows(self) -> int:
        v = ctypes.c_int()
        _check(lib().oqg_get_vty(self.h, ctypes.byref(v)), "oqg_get_vty")
        return v.value

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(lib().oqg_stream(self.h, ctypes.byref(s)), "oqg_stream")
        return s.value or 0

    def launch_floor(self, nsteps: int = 16) -> float:
        """Device microseconds per step of the step chain's launches with no work."""
        v = ctypes.c_double()
        _check(lib().oqg_launch_floor(self.h, int(nsteps), ctypes.byref(v)), "oqg_launch_floor")
        return v.value

    def step_launches(self) -> int:
        """Kernel launches of one model step (4, or 5 for wide boxes)."""
        v = ctypes.c_int()
        _check(lib().oqg_step_launches(self.h, ctypes.byref(v)), "oqg_step_launches")
        return v.value


def init_qg(basin: Basin) -> QG:
    """init_qg (qg.F90:60-103): modes, Helmholtz tables, homogeneous solutions."""
    return QG(basin)


def step_qg(tdt: float, ent, wekp, txis: float, txin: float, qg: QG):
    """step_qg (core.F90:16-33): one QG step with the given forcing."""
    qg.set_forcing(wekp, ent, txis, txin)
    qg.step(tdt, 1)


def suppress_comp_mode(qg: QG):
    """suppress_comp_mode (driver.F90:174-189)."""
    qg.suppress()


def ekman_from_tau(basin: Basin, taux, tauy):
    """ekman_from_tau (ekman.F90:53-83): (wekp, txis, txin) of a stress field."""
    prm = basin.to_c()
    taux = _f64(taux, basin.shape2)
    tauy = _f64(tauy, basin.shape2)
    w = np.empty(basin.shape2)
    ts, tn = ctypes.c_double(0.0), ctypes.c_double(0.0)
    _check(lib().oqg_ekman_from_tau(ctypes.byref(prm), _p(taux), _p(tauy), _p(w),
                                    ctypes.cast(ctypes.byref(ts), _dp),
                                    ctypes.cast(ctypes.byref(tn), _dp)), "oqg_ekman_from_tau")
    return w, ts.value, tn.value


class Ensemble:
    """Many basins of uneven size stepped together: one launch per phase of
    the step for all members (oqg_ensemble_*).  Members share nl, precision
    and kind (all boxes or all channels)."""

    def __init__(self, members):
        self.members = list(members)
        self._prm = [b.to_c() for b in self.members]
        arr = (type(self._prm[0]) * len(self._prm))(*self._prm)
        self._arr = arr
        e = ctypes.c_void_p()
        _check(lib().oqg_ensemble_create(ctypes.cast(arr, ctypes.c_void_p), len(self._prm), ctypes.byref(e)),
               "oqg_ensemble_create")
        self.e = e

    def close(self):
        if getattr(self, "e", None):
            lib().oqg_ensemble_destroy(self.e)
            self.e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.members)

    def set_state(self, i: int, p, pm):
        b = self.members[i]
        p, pm = _f64(p, b.shape3), _f64(pm, b.shape3)
        _check(lib().oqg_ensemble_set_state(self.e, i, _p(p), _p(pm)), "oqg_ensemble_set_state")

    def set_forcing(self, i: int, wekp=None, ent=None, txis=0.0, txin=0.0):
        b = self.members[i]
        wekp = _f64(wekp, b.shape2)
        ent = _f64(ent, (b.nl - 1,) + b.shape2) if ent is not None else None
        _check(lib().oqg_ensemble_set_forcing(self.e, i, _p(wekp), _p(ent), float(txis), float(txin)),
               "oqg_ensemble_set_forcing")

    def get_state(self, i: int):
        sh = self.members[i].shape3
        p, pm, q, qm = (np.empty(sh) for _ in range(4))
        _check(lib().oqg_ensemble_get_state(self.e, i, _p(p), _p(pm), _p(q), _p(qm)), "oqg_ensemble_get_state")
        return p, pm, q, qm

    def step(self, tdt, nsteps: int = 1):
        """tdt: one value for all members or one per member."""
        t = np.broadcast_to(np.asarray(tdt, dtype=np.float64), (len(self.members),)).copy()
        self._tdt = t
        _check(lib().oqg_ensemble_step(self.e, _p(t), int(nsteps)), "oqg_ensemble_step")

    def sync(self):
        _check(lib().oqg_ensemble_sync(self.e), "oqg_ensemble_sync")

    def autotune(self, tdt, nsteps: int = 10):
        """One vorticity tile height for all members, measured on the device
        from the members' current states (restored afterwards); returns
        (height, {height: ms per ensemble step})."""
        t = np.broadcast_to(np.asarray(tdt, dtype=np.float64), (len(self.members),)).copy()
        best = ctypes.c_int()
        ms = np.full(18, np.nan)
        _check(lib().oqg_ensemble_autotune(self.e, _p(t), int(nsteps), ctypes.byref(best), _p(ms)),
               "oqg_ensemble_autotune")
        return best.value, {v: float(ms[v]) for v in range(8, 18) if np.isfinite(ms[v])}

    def stream(self) -> int:
        s = ctypes.c_void_p()
        _check(lib().oqg_ensemble_stream(self.e, ctypes.byref(s)), "oqg_ensemble_stream")
        return s.value or 0


class OceanMixedLayer:
    """The ocean mixed layer of a closed basin on the device (step_oml,
    omlsubs.F90:69-119) coupled to a QG handle: `forcing(taux, tauy, fnetoc,
    compute_ent, tdto)` runs ekman_from_tau and step_oml and leaves wekp and
    ent in the handle's forcing for its next step (driver.F90:95-107).
    Arrays are numpy FP64: wind stress (nyp, nxp), T-grid fields (nyt, nxt)."""

    def __init__(self, qg: QG, hm: float, rho_cp: float, t1_rel: float, dt_12: float, st2d: float = 0.0,
                 st4d: float = 0.0, ycexp: float = 1.0, fluxn: bool = False, fluxs: bool = False,
                 nval: float = 0.0, sval: float = 0.0):
        self.qg = qg
        self._prm = OqgOmlParams(hm, rho_cp, t1_rel, dt_12, st2d, st4d, ycexp, int(fluxn), int(fluxs), nval, sval)
        h = ctypes.c_void_p()
        _check(lib().oqg_oml_create(qg.h, ctypes.byref(self._prm), ctypes.byref(h)), "oqg_oml_create")
        self.h = h
        self.tshape = (qg.b.nyp - 1, qg.b.nxp - 1)

    def close(self):
        # the mixed layer's buffers are freed without touching the QG handle,
        # so this is safe before or after the handle's close()
        if getattr(self, "h", None) is not None and self.h.value:
            lib().oqg_oml_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_sst(self, sst, sstm):
        a, am = _f64(sst, self.tshape), _f64(sstm, self.tshape)
        _check(lib().oqg_oml_set_sst(self.h, a.ctypes.data, am.ctypes.data), "oqg_oml_set_sst")

    def get_sst(self):
        a, am = np.empty(self.tshape), np.empty(self.tshape)
        _check(lib().oqg_oml_get_sst(self.h, a.ctypes.data, am.ctypes.data), "oqg_oml_get_sst")
        return a, am

    def couple(self, aml, raoro: float):
        """Links the atmospheric mixed layer for xforc() and
        compute_forcing() (oqg_oml_couple); aml None unlinks."""
        _check(lib().oqg_oml_couple(self.h, None if aml is None else aml.h, float(raoro)), "oqg_oml_couple")
        self._aml = aml          # keeps the atmosphere alive while coupled

    def tau_udiff(self, on: bool = True):
        """tau_udiff: the coupled stress follows the atmosphere-ocean
        velocity difference (oqg_oml_tau_udiff)."""
        _check(lib().oqg_oml_tau_udiff(self.h, int(bool(on))), "oqg_oml_tau_udiff")

    def compute_forcing(self, rad: OqgRadCoeffs):
        """Both mixed layers' net heat fluxes on the device (compute_forcing,
        forcing.F90:18-99), held for forcing() calls with fnet None."""
        _check(lib().oqg_compute_forcing(self.h, ctypes.byref(rad)), "oqg_compute_forcing")

    def get_fluxes(self):
        """The held fluxes: fnetoc (nyt, nxt) and, when coupled, the
        atmosphere's fnetat (None otherwise)."""
        fo = np.empty(self.tshape)
        aml = getattr(self, "_aml", None)
        fa = np.empty(aml.tshape) if aml is not None else None
        _check(lib().oqg_get_fluxes(self.h, fo.ctypes.data, None if fa is None else fa.ctypes.data),
               "oqg_get_fluxes")
        return fo, fa

    def forcing(self, taux, tauy, fnetoc, compute_ent: bool, tdto: float):
        """taux = tauy = None: the stress xforc() last computed; fnetoc None:
        the flux compute_forcing() last computed."""
        b = self.qg.b
        if taux is None and tauy is None:
            tx = ty = None
        else:
            tx, ty = _f64(taux, b.shape2), _f64(tauy, b.shape2)
        fn = None if fnetoc is None else _f64(fnetoc, self.tshape)
        _check(lib().oqg_ocean_forcing(self.h, None if tx is None else tx.ctypes.data,
                                       None if ty is None else ty.ctypes.data, None if fn is None else fn.ctypes.data,
                                       int(compute_ent), float(tdto)), "oqg_ocean_forcing")


def xforc(aml, oml=None):
    """Both basins' wind stress from the atmosphere's lagged layer-1 pressure
    on the device (xforc, windstress.F90:102-148), held for the forcing()
    calls with no stress: the atmosphere's, and the ocean's through the
    bicubic interpolation when oml (coupled to aml) is given."""
    _check(lib().oqg_xforc(aml.h, None if oml is None else oml.h), "oqg_xforc")


def get_forcing(qg: QG):
    """The handle's forcing (wekp (nyp, nxp), ent (nl-1, nyp, nxp))."""
    b = qg.b
    w, e = np.empty(b.shape2), np.empty((b.nl - 1,) + b.shape2)
    _check(lib().oqg_get_forcing(qg.h, _p(w), _p(e)), "oqg_get_forcing")
    return w, e


class AtmosMixedLayer:
    """The atmospheric mixed layer of a channel on the device (step_aml,
    amlsubs.F90:184-326) coupled to a QG handle: `forcing(taux, tauy, fnetat,
    compute_ent, tdta)` runs ekman_from_tau and step_aml and leaves wekp,
    txis, txin and ent in the handle's forcing (driver.F90:113-143).  The
    radiation-derived inputs (aface, bface, dface, xc1ast, fnetat) come from
    the caller.  Arrays are numpy FP64: stress and dtop (nyp, nxp), T-grid
    fields (nyt, nxt)."""

    def __init__(self, qg: QG, xc1ast, dtop=None, *, hm, rho_cp, t1_rel, dt_12, hmamin, hmadmp, xcexp,
                 at2d, at4d, ahmd, aface, bface, dface, cdat=1.3e-3):
        from .params import OQG_MAX_NL
        self.qg = qg
        b = qg.b
        self.tshape = (b.nyp - 1, b.nxp - 1)
        af = (ctypes.c_double * OQG_MAX_NL)(*([float(a) for a in aface] + [0.0] * (OQG_MAX_NL - len(aface))))
        self._prm = OqgAmlParams(hm, rho_cp, t1_rel, dt_12, hmamin, hmadmp, xcexp, at2d, at4d, ahmd, bface, dface,
                                 cdat, af)
        xc = _f64(xc1ast, self.tshape)
        dt = _f64(dtop, b.shape2) if dtop is not None else None
        h = ctypes.c_void_p()
        _check(lib().oqg_aml_create(qg.h, ctypes.byref(self._prm), xc.ctypes.data,
                                    None if dt is None else dt.ctypes.data, ctypes.byref(h)), "oqg_aml_create")
        self.h = h

    def close(self):
        # freed without touching the QG handle: safe before or after its close()
        if getattr(self, "h", None) is not None and self.h.value:
            lib().oqg_aml_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, ast, astm, hmixa, hmixam):
        a = [_f64(x, self.tshape) for x in (ast, astm, hmixa, hmixam)]
        _check(lib().oqg_aml_set_state(self.h, *[x.ctypes.data for x in a]), "oqg_aml_set_state")

    def get_state(self):
        a = [np.empty(self.tshape) for _ in range(4)]
        _check(lib().oqg_aml_get_state(self.h, *[x.ctypes.data for x in a]), "oqg_aml_get_state")
        return a

    def forcing(self, taux, tauy, fnetat, compute_ent: bool, tdta: float):
        """taux = tauy = None: the stress xforc() last computed on the
        device; fnetat None: the flux compute_forcing() last computed."""
        b = self.qg.b
        if taux is None and tauy is None:
            tx = ty = None
        else:
            tx, ty = _f64(taux, b.shape2), _f64(tauy, b.shape2)
        fn = None if fnetat is None else _f64(fnetat, self.tshape)
        _check(lib().oqg_atmos_forcing(self.h, None if tx is None else tx.ctypes.data,
                                       None if ty is None else ty.ctypes.data, None if fn is None else fn.ctypes.data,
                                       int(compute_ent), float(tdta)), "oqg_atmos_forcing")
