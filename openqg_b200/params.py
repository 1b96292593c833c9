"""Basin parameters and the synthetic workloads of the QG core.

`OqgParams` mirrors `oqg_params` in include/oqg.h (the fields of init_qg,
src/qg/qg.F90:60-70, plus the box geometry of src/glam/box.F90:11-41).
`Basin` is the Python-side description of one basin; the `ocean_*` and
`atmos_*` builders give the parameter sets of the benchmark workloads:

* double gyre ocean: 3 layers of 350/750/2900 m, reduced gravities
  0.05/0.025 m/s^2, f0 = 9.37e-5 1/s, beta = 1.75e-11 1/(m s), biharmonic
  ah4 = 2e10 m^4/s, bottom Ekman layer 2 m, no-slip walls (bcco = 1e20),
  dz_sign = -1, tau_sign = +1 and topography/drag in the bottom layer
  (basin.F90:36,62; topog.F90:52-56);
* atmosphere channel: 3 layers of 2000/3000/4000 m, reduced gravities
  1.2/0.4 m/s^2, ah4 = 2e13, bcco = 1, no bottom drag, dz_sign = +1,
  tau_sign = -1 and k_topo = 1 (data/basin/atm_dg.cdl).

Inputs are seeded and synthetic (no reference data files exist): the
initial stream function is Gaussian noise on the interior, low-passed to DST
modes k, l < 8 and scaled to a standard deviation of 1e3 m^2/s; the wind is
the analytic double-gyre stress tau_x = -A cos(2 pi y / Ly) / rho0.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

OQG_MAX_NL = 8
OQG_FP64 = 0
OQG_MIXED = 1

STATUS = {
    0: "OQG_OK", 1: "OQG_EINVAL", 2: "OQG_ECUDA", 3: "OQG_ENAN",
    4: "OQG_ETIMEOUT", 5: "OQG_EUNSUPPORTED", 6: "OQG_ESETUP", 7: "OQG_ENODEV",
    8: "OQG_ESCRATCH",
}

_D8 = ctypes.c_double * OQG_MAX_NL


class OqgOmlParams(ctypes.Structure):
    """ctypes mirror of `oqg_oml_params` (include/oqg.h): the ocean mixed
    layer's parameters (init_ocean_ml, omlsubs.F90:27-67)."""
    _fields_ = [
        ("hm", ctypes.c_double), ("rho_cp", ctypes.c_double), ("t1_rel", ctypes.c_double),
        ("dt_12", ctypes.c_double), ("st2d", ctypes.c_double), ("st4d", ctypes.c_double),
        ("ycexp", ctypes.c_double), ("fluxn", ctypes.c_int), ("fluxs", ctypes.c_int),
        ("nval", ctypes.c_double), ("sval", ctypes.c_double),
    ]


class OqgAmlParams(ctypes.Structure):
    """ctypes mirror of `oqg_aml_params` (include/oqg.h): the atmospheric
    mixed layer's parameters (init_atmos_ml, amlsubs.F90:61-131)."""
    _fields_ = [(n, ctypes.c_double) for n in ("hm", "rho_cp", "t1_rel", "dt_12", "hmamin", "hmadmp", "xcexp",
                                               "at2d", "at4d", "ahmd", "bface", "dface", "cdat")] + \
        [("aface", ctypes.c_double * OQG_MAX_NL)]


class OqgRadCoeffs(ctypes.Structure):
    """ctypes mirror of `oqg_rad_coeffs` (include/oqg.h): the radiation
    coefficients compute_forcing reads (radiate_type, radsubs.F90:15-54)."""
    _fields_ = [(n, ctypes.c_double) for n in ("fspco", "xlamda", "d0up", "dmdown", "dup0", "aup00", "adown10",
                                               "adown11")]


class OqgRadParams(ctypes.Structure):
    """ctypes mirror of `oqg_rad_params` (include/oqg.h): load_rad's inputs."""
    _fields_ = [("fsbar", ctypes.c_double), ("fspamp", ctypes.c_double), ("gamma", ctypes.c_double),
                ("xlamda", ctypes.c_double), ("zopt", ctypes.c_double * (OQG_MAX_NL + 1)),
                ("tabsat", ctypes.c_double * OQG_MAX_NL)]


class OqgRadState(ctypes.Structure):
    """ctypes mirror of `oqg_rad_state` (include/oqg.h): radiat's results."""
    _fields_ = [("c", OqgRadCoeffs), ("aup", (ctypes.c_double * OQG_MAX_NL) * (OQG_MAX_NL + 1)),
                ("adown", (ctypes.c_double * OQG_MAX_NL) * OQG_MAX_NL), ("dup", ctypes.c_double * (OQG_MAX_NL + 1)),
                ("rbetat", ctypes.c_double * OQG_MAX_NL), ("rbtmat", ctypes.c_double), ("rbtmoc", ctypes.c_double),
                ("atm_tmbar", ctypes.c_double), ("ocn_tmbar", ctypes.c_double)]


class OqgParams(ctypes.Structure):
    """ctypes mirror of `oqg_params` (include/oqg.h)."""
    _fields_ = [
        ("nxp", ctypes.c_int), ("nyp", ctypes.c_int), ("nl", ctypes.c_int),
        ("cyclic", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("fnot", ctypes.c_double), ("beta", ctypes.c_double),
        ("dz_sign", ctypes.c_int), ("tau_sign", ctypes.c_int),
        ("h", _D8), ("gp", _D8), ("ah2", _D8), ("ah4", _D8),
        ("bcco", ctypes.c_double), ("delek", ctypes.c_double),
        ("rho", ctypes.c_double),
        ("k_topo", ctypes.c_int), ("precision", ctypes.c_int),
        ("suppress_period", ctypes.c_int),
        ("ddyn", ctypes.POINTER(ctypes.c_double)),
    ]


class QgMonitor(ctypes.Structure):
    """oqg_qg_monitor of include/oqg.h: the qg_diagno record
    (qg_monitor.F90:219-383)."""
    _fields_ = [("tsec", ctypes.c_double), ("wepm", ctypes.c_double), ("wapm", ctypes.c_double),
                ("entm", ctypes.c_double), ("enam", ctypes.c_double),
                ("etam", ctypes.c_double * OQG_MAX_NL), ("et2m", ctypes.c_double * OQG_MAX_NL),
                ("pket", ctypes.c_double * OQG_MAX_NL), ("pken", ctypes.c_double), ("utau", ctypes.c_double),
                ("pavg", ctypes.c_double * OQG_MAX_NL), ("qavg", ctypes.c_double * OQG_MAX_NL),
                ("ah2d", ctypes.c_double * OQG_MAX_NL), ("ah4d", ctypes.c_double * OQG_MAX_NL),
                ("ekei", ctypes.c_double * OQG_MAX_NL), ("val", ctypes.c_double * OQG_MAX_NL),
                ("pos", ctypes.c_int * OQG_MAX_NL), ("circ", ctypes.c_double * OQG_MAX_NL),
                ("ctot", ctypes.c_double), ("btdg", ctypes.c_double),
                ("sfmin", ctypes.c_double * OQG_MAX_NL), ("sfmax", ctypes.c_double * OQG_MAX_NL),
                ("ermas", ctypes.c_double * OQG_MAX_NL), ("emfr", ctypes.c_double * OQG_MAX_NL)]

    def as_dict(self, nl: int) -> dict:
        out = {}
        for name, typ in self._fields_:
            v = getattr(self, name)
            if hasattr(typ, "_length_"):
                n = nl - 1 if name in ("etam", "et2m", "pket", "ermas", "emfr") else nl
                out[name] = np.array(v[:n])
            else:
                out[name] = float(v)
        return out


@dataclass
class Basin:
    """One QG basin (the `box_type`, `topog_type` and `qg_type` parameters)."""
    nxp: int
    nyp: int
    dx: float
    dy: float
    h: Sequence[float]
    gp: Sequence[float]
    fnot: float = 9.37e-5
    beta: float = 1.75e-11
    cyclic: bool = False
    dz_sign: int = -1
    tau_sign: int = 1
    ah2: Optional[Sequence[float]] = None
    ah4: Optional[Sequence[float]] = None
    bcco: float = 1.0e20
    delek: float = 2.0
    rho: float = 1.0e3
    k_topo: Optional[int] = None          # 1-based; default from dz_sign
    precision: int = OQG_FP64
    suppress_period: int = 25
    ddyn: Optional[np.ndarray] = None     # (nxp, nyp) Fortran order
    _keep: list = field(default_factory=list, repr=False)

    @property
    def nl(self) -> int:
        return len(self.h)

    @property
    def shape3(self):
        """(nl, nyp, nxp): C-order view of a Fortran (nxp, nyp, nl) array."""
        return (self.nl, self.nyp, self.nxp)

    @property
    def shape2(self):
        return (self.nyp, self.nxp)

    @property
    def yprel(self) -> np.ndarray:
        yl = (self.nyp - 1) * self.dy
        return -0.5 * yl + np.arange(self.nyp) * self.dy

    def ktopo(self) -> int:
        if self.k_topo is not None:
            return self.k_topo
        return 1 if self.dz_sign == 1 else self.nl   # topog.F90:52-56

    def to_c(self) -> OqgParams:
        nl = self.nl
        if not 2 <= nl <= OQG_MAX_NL:
            raise ValueError("nl must be in [2, %d]" % OQG_MAX_NL)
        p = OqgParams()
        p.nxp, p.nyp, p.nl = self.nxp, self.nyp, nl
        p.cyclic = 1 if self.cyclic else 0
        p.dx, p.dy, p.fnot, p.beta = self.dx, self.dy, self.fnot, self.beta
        p.dz_sign, p.tau_sign = self.dz_sign, self.tau_sign
        ah2 = list(self.ah2) if self.ah2 is not None else [0.0] * nl
        ah4 = list(self.ah4) if self.ah4 is not None else [0.0] * nl
        for k in range(nl):
            p.h[k] = self.h[k]
            p.ah2[k] = ah2[k]
            p.ah4[k] = ah4[k]
        for k in range(nl - 1):
            p.gp[k] = self.gp[k]
        p.bcco, p.delek, p.rho = self.bcco, self.delek, self.rho
        p.k_topo = self.ktopo()
        p.precision = self.precision
        p.suppress_period = self.suppress_period
        if self.ddyn is not None:
            d = np.ascontiguousarray(self.ddyn, dtype=np.float64)
            if d.size != self.nxp * self.nyp:
                raise ValueError("ddyn must have nxp*nyp values")
            self._keep[:] = [d]
            p.ddyn = d.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        else:
            p.ddyn = None
        return p


def ocean_double_gyre(n: int = 129, dx: float = 20.0e3, ah4: float = 2.0e10,
                      precision: int = OQG_FP64, suppress_period: int = 25) -> Basin:
    """Ocean-only 3-layer double gyre on an n x n p-grid (closed box)."""
    return Basin(nxp=n, nyp=n, dx=dx, dy=dx, h=[350.0, 750.0, 2900.0],
                 gp=[0.05, 0.025], fnot=9.37e-5, beta=1.75e-11, cyclic=False,
                 dz_sign=-1, tau_sign=1, ah2=[0.0] * 3, ah4=[ah4] * 3,
                 bcco=1.0e20, delek=2.0, rho=1.0e3, precision=precision,
                 suppress_period=suppress_period)


def atmos_channel(nxp: int = 193, nyp: int = 97, dx: float = 80.0e3,
                  precision: int = OQG_FP64, suppress_period: int = 100) -> Basin:
    """3-layer atmosphere in a zonally periodic channel."""
    return Basin(nxp=nxp, nyp=nyp, dx=dx, dy=dx, h=[2000.0, 3000.0, 4000.0],
                 gp=[1.2, 0.4], fnot=9.37e-5, beta=1.75e-11, cyclic=True,
                 dz_sign=1, tau_sign=-1, ah2=[0.0] * 3, ah4=[2.0e13] * 3,
                 bcco=1.0, delek=0.0, rho=1.0, k_topo=1, precision=precision,
                 suppress_period=suppress_period)


def _dst1_matrix(n: int) -> np.ndarray:
    """Orthogonal DST-I matrix of size n (used only to build initial states)."""
    j = np.arange(1, n + 1)
    return np.sqrt(2.0 / (n + 1)) * np.sin(np.pi * np.outer(j, j) / (n + 1))


def initial_psi(b: Basin, seed: int = 0, kmax: int = 8, std: float = 1.0e3) -> np.ndarray:
    """Seeded low-passed noise stream function (nl, nyp, nxp), zero on walls.

    Interior values are i.i.d. N(0,1), low-passed to sine modes k, l < kmax by
    a 2-D DST-I, and scaled to standard deviation `std` (m^2/s) per layer.
    For a channel the x-direction low-pass uses a real FFT instead.
    """
    rng = np.random.default_rng(seed)
    out = np.zeros(b.shape3)
    nyi = b.nyp - 2
    Sy = _dst1_matrix(nyi)
    for k in range(b.nl):
        if b.cyclic:
            nx = b.nxp - 1
            w = rng.standard_normal((nyi, nx))
            c = Sy @ w
            c[kmax - 1:, :] = 0.0
            f = np.fft.rfft(c, axis=1)
            f[:, kmax:] = 0.0
            lo = np.fft.irfft(f, n=nx, axis=1)
            lo = Sy @ lo
            lo *= std / max(lo.std(), 1e-300)
            out[k, 1:-1, :nx] = lo
            out[k, 1:-1, nx] = lo[:, 0]
        else:
            nxi = b.nxp - 2
            Sx = _dst1_matrix(nxi)
            w = rng.standard_normal((nyi, nxi))
            c = Sy @ w @ Sx
            c[kmax - 1:, :] = 0.0
            c[:, kmax - 1:] = 0.0
            lo = Sy @ c @ Sx
            lo *= std / max(lo.std(), 1e-300)
            out[k, 1:-1, 1:-1] = lo
    return out


def double_gyre_tau(b: Basin, amp: float = 0.1, rho0: float = 1.0e3):
    """Kinematic stress (taux, tauy) of shape (nyp, nxp): -amp cos(2 pi y/Ly)/rho0."""
    yl = (b.nyp - 1) * b.dy
    y = np.arange(b.nyp) * b.dy
    tx = -amp * np.cos(2.0 * np.pi * y / yl) / rho0
    taux = np.repeat(tx[:, None], b.nxp, axis=1)
    tauy = np.zeros_like(taux)
    return taux, tauy


def fortran3(a: np.ndarray) -> np.ndarray:
    """(nl, nyp, nxp) C-order array -> contiguous buffer in Fortran (nxp,nyp,nl) order.

    A C-order (nl, nyp, nxp) array already has the memory layout of a
    Fortran (nxp, nyp, nl) array, so this only enforces dtype and contiguity.
    """
    return np.ascontiguousarray(a, dtype=np.float64)
