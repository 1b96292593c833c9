"""Restart files: the reference's netCDF restart (save_qg / restart_qg,
src/state.F90:29-112) and the exact device-state checkpoint."""
import os

import numpy as np
import pytest
from scipy.io import netcdf_file

from openqg_b200.params import atmos_channel, double_gyre_tau, initial_psi, ocean_double_gyre
from openqg_b200.restart import restart_qg, save_qg


def test_save_qg_writes_the_reference_layout(tmp_path):
    b = ocean_double_gyre(33)
    p = b.fnot * initial_psi(b, 1)
    pm = 0.5 * p
    path = os.path.join(tmp_path, "lastday.nc")
    save_qg(path, b, p, pm)
    f = netcdf_file(path, "r", mmap=False)
    assert f.version_byte == 1                       # classic format (NF90_CLOBBER)
    assert f.dimensions == {"nxp": 33, "nyp": 33, "nl": 3}
    assert f.variables["p"].dimensions == ("nl", "nyp", "nxp")
    assert f.variables["p"].units == b"Current pressure"
    assert f.variables["pm"].units == b"Previous pressure"
    assert f.variables["x"].units == b"km"
    assert np.allclose(f.variables["x"][:], np.arange(33) * b.dx * 1e-3)
    f.close()
    p2, pm2 = restart_qg(path, b)
    assert np.array_equal(p2, p) and np.array_equal(pm2, pm)


def test_restart_rejects_another_grid(tmp_path):
    b = atmos_channel(49, 25)
    path = os.path.join(tmp_path, "atm.nc")
    save_qg(path, b, np.zeros(b.shape3), np.zeros(b.shape3))
    with pytest.raises(ValueError):
        restart_qg(path, atmos_channel(97, 65))


@pytest.mark.gpu
def test_device_restart_and_exact_checkpoint(tmp_path, gpu_required):
    import oracle
    from openqg_b200.core import QG
    from openqg_b200.restart import restart_into, restore_state, save_state
    b = ocean_double_gyre(65)
    p = b.fnot * initial_psi(b, 3)
    w, ts, tn = oracle.ekman_from_tau(b, *double_gyre_tau(b))
    nc = os.path.join(tmp_path, "ocn.nc")
    save_qg(nc, b, p, p)
    g1, g2 = QG(b), QG(b)
    for g in (g1, g2):
        g.set_forcing(w, None, ts, tn)
    g1.set_state(p, p)
    restart_into(nc, g2)                       # the reference's restart path
    g1.step(3600.0, 5)
    g2.step(3600.0, 5)
    for a, c in zip(g1.get_state(), g2.get_state()):
        assert np.array_equal(a, c)
    # exact continuation through a full-state checkpoint, across parities
    ck = os.path.join(tmp_path, "state.npz")
    save_state(ck, g1)
    g1.step(3600.0, 6)
    g3 = QG(b)
    g3.set_forcing(w, None, ts, tn)
    g3.step(3600.0, 1)                         # a handle at the other parity
    restore_state(ck, g3)
    g3.step(3600.0, 6)
    assert g3.step_index() == g1.step_index() == 11
    for a, c in zip(g1.get_state(), g3.get_state()):
        assert np.array_equal(a, c)
