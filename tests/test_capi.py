"""The C-ABI library loads and exports every entry point include/oqg.h declares
(no GPU needed; no compute call is made without a device)."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from openqg_b200 import build as oqg_build
from openqg_b200 import core
from openqg_b200.params import OqgParams, atmos_channel, double_gyre_tau, ocean_double_gyre
from tests.conftest import has_gpu

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "oqg.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(oqg_\w+)\s*\(", src, flags=re.M)))


@pytest.fixture(scope="module")
def liboqg():
    oqg_build.build()
    return core.lib()


def test_header_declares_the_step_boundary():
    names = declared_functions()
    for must in ("oqg_create", "oqg_step", "oqg_set_state", "oqg_get_state", "oqg_set_forcing",
                 "oqg_suppress", "oqg_destroy", "oqg_ensemble_step"):
        assert must in names


def test_library_exports_every_declared_symbol(liboqg):
    missing = [n for n in declared_functions() if not hasattr(liboqg, n)]
    assert not missing, missing


def test_params_struct_layout_matches_header():
    # offsets fixed by the C struct in include/oqg.h (x86-64 ABI)
    assert OqgParams.h.offset == 56
    assert OqgParams.bcco.offset == 56 + 4 * 64
    assert ctypes.sizeof(OqgParams) == 56 + 4 * 64 + 24 + 16 + 8


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_create_without_device_reports_enodev(liboqg):
    prm = ocean_double_gyre(33).to_c()
    h = ctypes.c_void_p()
    rc = liboqg.oqg_create(ctypes.byref(prm), ctypes.byref(h))
    assert rc == 7 and not h.value
    assert b"device" in liboqg.oqg_last_error()


def test_create_rejects_bad_params(liboqg):
    b = ocean_double_gyre(33)
    prm = b.to_c()
    prm.nl = 9
    h = ctypes.c_void_p()
    assert liboqg.oqg_create(ctypes.byref(prm), ctypes.byref(h)) in (1, 5)
    assert liboqg.oqg_create(None, ctypes.byref(h)) == 1


def test_ekman_from_tau_matches_oracle(liboqg):
    """Init-time host routine of the library (ekman.F90:53-83)."""
    for b in (ocean_double_gyre(65), atmos_channel(49, 25)):
        taux, tauy = double_gyre_tau(b)
        tauy = tauy + 1e-5 * np.cos(np.arange(b.nxp) * 0.3)[None, :]
        wg, sg, ng = core.ekman_from_tau(b, taux, tauy)
        wo, so, no = oracle.ekman_from_tau(b, taux, tauy)
        assert np.array_equal(wg, wo)
        assert sg == so and ng == no


def test_ensemble_create_checks_members_before_any_device_call(liboqg):
    import ctypes
    from openqg_b200.params import atmos_channel, ocean_double_gyre
    a, c = ocean_double_gyre(33), atmos_channel(49, 25)
    c.h = [2000.0, 3000.0]
    c.gp = [1.2]
    two = [a.to_c(), c.to_c()]
    arr = (type(two[0]) * 2)(*two)
    e = ctypes.c_void_p()
    # members of different nl: OQG_EINVAL
    assert liboqg.oqg_ensemble_create(ctypes.cast(arr, ctypes.c_void_p), 2, ctypes.byref(e)) == 1
    # a box with a channel: OQG_EUNSUPPORTED
    b3 = atmos_channel(49, 25).to_c()
    arr2 = (type(b3) * 2)(a.to_c(), b3)
    assert liboqg.oqg_ensemble_create(ctypes.cast(arr2, ctypes.c_void_p), 2, ctypes.byref(e)) == 5
    assert not e.value


def test_oml_params_struct_layout_matches_header():
    from openqg_b200.params import OqgOmlParams
    # seven doubles, two ints, two doubles (x86-64 ABI)
    assert OqgOmlParams.fluxn.offset == 56
    assert OqgOmlParams.nval.offset == 64
    assert ctypes.sizeof(OqgOmlParams) == 80


def test_added_entry_points_reject_null_arguments(liboqg):
    """The adjoint, state-slot, autotuning and mixed-layer entry points check
    their arguments before any device call."""
    L = liboqg
    assert L.oqg_adj_set(None, None, None, None, None, None, None) == 1
    assert L.oqg_adj_get(None, None, None, None, None, None, None, None) == 1
    assert L.oqg_adj_step(None, None, ctypes.c_double(1.0), ctypes.c_longlong(1)) == 1
    assert L.oqg_adj_segment(None, None, None, ctypes.c_size_t(0), 1, ctypes.c_double(1.0),
                             ctypes.c_longlong(1)) == 1
    assert L.oqg_adj_initial(None, None, None) == 1
    assert L.oqg_state_bytes(None, None, None) == 1
    assert L.oqg_state_save(None, None) == 1
    assert L.oqg_state_load(None, None) == 1
    assert L.oqg_pq_save(None, None) == 1
    assert L.oqg_autotune(None, ctypes.c_double(1.0), 4, None, None) == 1
    assert L.oqg_ensemble_autotune(None, None, 4, None, None) == 1
    assert L.oqg_get_vty(None, None) == 1
    assert L.oqg_oml_create(None, None, None) == 1
    assert L.oqg_oml_destroy(None) == 0
    assert L.oqg_oml_set_sst(None, None, None) == 1
    assert L.oqg_oml_get_sst(None, None, None) == 1
    assert L.oqg_ocean_forcing(None, None, None, None, 1, ctypes.c_double(1.0)) == 1
    assert L.oqg_get_forcing(None, None, None) == 1
    assert L.oqg_aml_create(None, None, None, None, None) == 1
    assert L.oqg_aml_destroy(None) == 0
    assert L.oqg_aml_set_state(None, None, None, None, None) == 1
    assert L.oqg_aml_get_state(None, None, None, None, None) == 1
    assert L.oqg_atmos_forcing(None, None, None, None, 1, ctypes.c_double(1.0)) == 1
    assert L.oqg_oml_couple(None, None, ctypes.c_double(1.2e-3)) == 1
    assert L.oqg_xforc(None, None) == 1
    assert L.oqg_oml_tau_udiff(None, 1) == 1
    assert L.oqg_compute_forcing(None, None) == 1
    assert L.oqg_get_fluxes(None, None, None) == 1
    assert L.oqg_radiat(3, None, ctypes.c_double(1.0), ctypes.c_double(1.0), None, None) == 1
    assert L.oqg_entrain_coeff(3, ctypes.c_double(1.0), ctypes.c_double(1.0), None, None, None, None) == 1
    assert L.oqg_zonal_temp(1, *([ctypes.c_double(1.0)] * 6), None) == 1


def test_rad_coeffs_struct_layout_matches_header():
    from openqg_b200.params import OqgRadCoeffs
    assert ctypes.sizeof(OqgRadCoeffs) == 8 * 8
    assert OqgRadCoeffs.adown11.offset == 7 * 8
    from openqg_b200.params import OqgRadParams, OqgRadState
    assert ctypes.sizeof(OqgRadParams) == (4 + 9 + 8) * 8
    assert OqgRadParams.tabsat.offset == (4 + 9) * 8
    assert OqgRadState.dup.offset == (8 + 9 * 8 + 8 * 8) * 8
    assert ctypes.sizeof(OqgRadState) == (8 + 9 * 8 + 8 * 8 + 9 + 8 + 4) * 8


def test_aml_params_struct_layout_matches_header():
    from openqg_b200.params import OqgAmlParams
    assert OqgAmlParams.aface.offset == 13 * 8
    assert ctypes.sizeof(OqgAmlParams) == 13 * 8 + 8 * 8
