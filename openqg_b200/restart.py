"""Restart files of the QG state.

`save_qg` / `restart_qg` read and write the reference's restart file
(src/state.F90:29-112): a classic-format netCDF file with dimensions
nxp, nyp, nl and double variables x(nxp), y(nyp) in km and p, pm
(nl, nyp, nxp in netCDF order, i.e. Fortran (nxp, nyp, nl)).  As in the
reference, the pressure variables carry their description in the `units`
attribute, and a restart sets p and pm only: q, qm and the constraints are
recomputed from them (init_pv and init_mass_constr / init_constraint, as
init_dynamic_state does, openqg.F90:233-243).

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
