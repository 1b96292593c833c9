"""Restart files of the QG state.

`save_qg` / `restart_qg` read and write the reference's restart file
(src/state.F90:29-112): a classic-format netCDF file with dimensions
nxp, nyp, nl and double variables x(nxp), y(nyp) in km and p, pm
(nl, nyp, nxp in netCDF order, i.e. Fortran (nxp, nyp, nl)).  As in the
reference, the pressure variables carry their description in the `units`
attribute, and a restart sets p and pm only: q, qm and the constraints are
recomputed from them (init_pv and init_mass_constr / init_constraint, as
init_dynamic_state does, openqg.F90:233-243).

`save_oml` / `restart_oml` and `save_aml` / `restart_aml` are the mixed
layers' restart files (state.F90:46-80, 114-178): dimensions nxt, nyt, the
T-point coordinates x, y in km, and sst, sstm (ocean) or ast, astm, hmixa,
hmixam (atmosphere), each (nyt, nxt) in netCDF order.  `restart_*_into`
loads one into a device mixed layer.

`save_state` / `restore_state` go further: every field of the device state
(p, pm, q, qm, the mass and momentum constraints and the step index), so a
restored handle continues bit for bit.  They use numpy's .npz format.
"""
from __future__ import annotations

import numpy as np
from scipy.io import netcdf_file

from .params import Basin


def _coords(b: Basin, x0: float = 0.0, y0: float = 0.0):
    xp = x0 + np.arange(b.nxp) * b.dx
    yp = y0 + np.arange(b.nyp) * b.dy
    return xp * 1.0e-3, yp * 1.0e-3          # m_to_km


def save_qg(path: str, b: Basin, p: np.ndarray, pm: np.ndarray, x0: float = 0.0, y0: float = 0.0) -> None:
    """save_qg (state.F90:88-112): p, pm of shape (nl, nyp, nxp)."""
    p = np.asarray(p, dtype=np.float64).reshape(b.shape3)
    pm = np.asarray(pm, dtype=np.float64).reshape(b.shape3)
    x, y = _coords(b, x0, y0)
    f = netcdf_file(path, "w", version=1)
    try:
        f.createDimension("nxp", b.nxp)
        f.createDimension("nyp", b.nyp)
        f.createDimension("nl", b.nl)
        vx = f.createVariable("x", "d", ("nxp",))
        vx.units = "km"
        vy = f.createVariable("y", "d", ("nyp",))
        vy.units = "km"
        vp = f.createVariable("p", "d", ("nl", "nyp", "nxp"))
        vp.units = "Current pressure"
        vpm = f.createVariable("pm", "d", ("nl", "nyp", "nxp"))
        vpm.units = "Previous pressure"
        vx[:] = x
        vy[:] = y
        vp[:] = p
        vpm[:] = pm
    finally:
        f.close()


def restart_qg(path: str, b: Basin):
    """restart_qg (state.F90:29-42): returns (p, pm), each (nl, nyp, nxp).
    Raises ValueError when the file's grid is not the basin's."""
    f = netcdf_file(path, "r", mmap=False)
    try:
        shape = (f.dimensions["nl"], f.dimensions["nyp"], f.dimensions["nxp"])
        if tuple(shape) != b.shape3:
            raise ValueError("restart grid %s does not match the basin %s" % (shape, b.shape3))
        p = np.array(f.variables["p"][:], dtype=np.float64)
        pm = np.array(f.variables["pm"][:], dtype=np.float64)
    finally:
        f.close()
    return p, pm


def restart_into(path: str, qg) -> None:
    """Reads a reference restart file into a device handle: set_state(p, pm)."""
    p, pm = restart_qg(path, qg.b)
    qg.set_state(p, pm)


def _tcoords(b: Basin, x0: float = 0.0, y0: float = 0.0):
    """T-point coordinates in km: xt(i) = xp(i) + dx/2 (box.F90:145-160)."""
    xt = x0 + (np.arange(b.nxp - 1) + 0.5) * b.dx
    yt = y0 + (np.arange(b.nyp - 1) + 0.5) * b.dy
    return xt * 1.0e-3, yt * 1.0e-3


def _save_t_fields(path: str, b: Basin, fields, x0: float, y0: float) -> None:
    tshape = (b.nyp - 1, b.nxp - 1)
    x, y = _tcoords(b, x0, y0)
    f = netcdf_file(path, "w", version=1)
    try:
        f.createDimension("nxt", tshape[1])
        f.createDimension("nyt", tshape[0])
        vx = f.createVariable("x", "d", ("nxt",))
        vx.units = "km"
        vy = f.createVariable("y", "d", ("nyt",))
        vy.units = "km"
        vx[:] = x
        vy[:] = y
        for name, desc, a in fields:
            v = f.createVariable(name, "d", ("nyt", "nxt"))
            v.units = desc
            v[:] = np.asarray(a, dtype=np.float64).reshape(tshape)
    finally:
        f.close()


def _read_t_fields(path: str, b: Basin, names):
    tshape = (b.nyp - 1, b.nxp - 1)
    f = netcdf_file(path, "r", mmap=False)
    try:
        shape = (f.dimensions["nyt"], f.dimensions["nxt"])
        if tuple(shape) != tshape:
            raise ValueError("restart T grid %s does not match the basin's %s" % (shape, tshape))
        return [np.array(f.variables[n][:], dtype=np.float64) for n in names]
    finally:
        f.close()


def save_oml(path: str, b: Basin, sst, sstm, x0: float = 0.0, y0: float = 0.0) -> None:
    """save_oml (state.F90:114-143): the ocean mixed layer's temperature at
    the current and previous level, T grid (nyt, nxt)."""
    _save_t_fields(path, b, [("sst", "Current mixed layer temp", sst),
                             ("sstm", "Previous mixed layer temp", sstm)], x0, y0)


def restart_oml(path: str, b: Basin):
    """restart_oml (state.F90:46-61): returns (sst, sstm)."""
    return tuple(_read_t_fields(path, b, ("sst", "sstm")))


def save_aml(path: str, b: Basin, ast, astm, hmixa, hmixam, x0: float = 0.0, y0: float = 0.0) -> None:
    """save_aml (state.F90:145-178): the atmospheric mixed layer's
    temperature and height at the current and previous level."""
    _save_t_fields(path, b, [("ast", "Current mixed layer temp", ast),
                             ("astm", "Previous mixed layer temp", astm),
                             ("hmixa", "Current mixed layer height", hmixa),
                             ("hmixam", "Previous mixed layer height", hmixam)], x0, y0)


def restart_aml(path: str, b: Basin):
    """restart_aml (state.F90:63-80): returns (ast, astm, hmixa, hmixam)."""
    return tuple(_read_t_fields(path, b, ("ast", "astm", "hmixa", "hmixam")))


def restart_oml_into(path: str, oml) -> None:
    """Reads an ocean mixed-layer restart file into a device mixed layer."""
    oml.set_sst(*restart_oml(path, oml.qg.b))


def restart_aml_into(path: str, aml) -> None:
    """Reads an atmospheric mixed-layer restart file into a device mixed layer."""
    aml.set_state(*restart_aml(path, aml.qg.b))


def save_state(path: str, qg) -> None:
    """The whole device state of a handle, for an exact continuation."""
    p, pm, q, qm = qg.get_state()
    c = qg.constraints()
    np.savez(path, p=p, pm=pm, q=q, qm=qm, step_index=np.int64(qg.step_index()),
             nxp=qg.b.nxp, nyp=qg.b.nyp, nl=qg.b.nl, **c)


def restore_state(path: str, qg) -> None:
    d = np.load(path)
    if (int(d["nxp"]), int(d["nyp"]), int(d["nl"])) != (qg.b.nxp, qg.b.nyp, qg.b.nl):
        raise ValueError("state file grid does not match the basin")
    qg.set_state_full(d["p"], d["pm"], d["q"], d["qm"], d["dpi"], d["dpip"],
                      d["cs"], d["cn"], d["csp"], d["cnp"])
    qg.set_step_index(int(d["step_index"]))
