"""Restart files: the reference's netCDF restart (save_qg / restart_qg,
src/state.F90:29-112) and the exact device-state checkpoint."""
import os

import numpy as np
import pytest
from scipy.io import netcdf_file

from openqg_b200.params import atmos_channel, double_gyre_tau, initial_psi, ocean_double_gyre
from openqg_b200.restart import restart_aml, restart_oml, restart_qg, save_aml, save_oml, save_qg


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


def test_mixed_layer_restarts_round_trip(tmp_path):
    """save_oml / restart_oml and save_aml / restart_aml (state.F90:46-80,
    114-178): T-grid dimensions nxt, nyt, the reference's variable names and
    descriptions, exact round trips."""
    rng = np.random.default_rng(3)
    bo, ba = ocean_double_gyre(33), atmos_channel(49, 25)
    to, ta = (bo.nyp - 1, bo.nxp - 1), (ba.nyp - 1, ba.nxp - 1)
    sst, sstm = rng.standard_normal(to), rng.standard_normal(to)
    po = os.path.join(tmp_path, "oml.nc")
    save_oml(po, bo, sst, sstm)
    f = netcdf_file(po, "r", mmap=False)
    assert f.dimensions == {"nxt": 32, "nyt": 32}
    assert f.variables["sst"].dimensions == ("nyt", "nxt")
    assert f.variables["sstm"].units == b"Previous mixed layer temp"
    assert np.allclose(f.variables["x"][:], (np.arange(32) + 0.5) * bo.dx * 1e-3)
    f.close()
    a, am = restart_oml(po, bo)
    assert np.array_equal(a, sst) and np.array_equal(am, sstm)
    fa = [rng.standard_normal(ta) for _ in range(4)]
    pa = os.path.join(tmp_path, "aml.nc")
    save_aml(pa, ba, *fa)
    f = netcdf_file(pa, "r", mmap=False)
    assert sorted(f.variables) == ["ast", "astm", "hmixa", "hmixam", "x", "y"]
    assert f.variables["hmixa"].units == b"Current mixed layer height"
    f.close()
    for got, want in zip(restart_aml(pa, ba), fa):
        assert np.array_equal(got, want)
    with pytest.raises(ValueError):
        restart_oml(po, ocean_double_gyre(65))


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
