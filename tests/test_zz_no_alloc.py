"""oqg_diag_noalloc: the diagnostics entry point whose scratch is a fixed
device array in the library, checked against oqg_diag through the C ABI.

Collected last (file name), so it also runs after every other test has used
the library on the same device.  Each case calls the entry point twice in a
row: the second call must find its completion counter cleared again.
"""
import ctypes

import numpy as np
import pytest

from openqg_b200.core import QG, OqgError, lib
from openqg_b200.params import OQG_MIXED, atmos_channel, initial_psi, ocean_double_gyre

# ekei is summed by rows first here and by strided threads in oqg_diag, so it
# agrees to rounding; the extrema and the circulation are the same operations.
EKEI_RTOL = 1e-12

CASES = [
    (ocean_double_gyre(129), 3600.0),
    (ocean_double_gyre(513, dx=10e3), 3600.0),
    (atmos_channel(193, 97), 360.0),
]
IDS = ["box129", "box513", "chan193x97"]


def _stepped(b, tdt, nsteps=3):
    g = QG(b)
    p = b.fnot * initial_psi(b, 5) * (30.0 if b.cyclic else 1.0)
    g.set_state(p, p)
    g.step(tdt, nsteps)
    return g


def _call(g):
    nl = g.b.nl
    out = [np.full(nl, np.nan) for _ in range(4)]
    dp = ctypes.POINTER(ctypes.c_double)
    rc = lib().oqg_diag_noalloc(g.h, *(a.ctypes.data_as(dp) for a in out))
    return rc, dict(zip(("ekei", "sfmin", "sfmax", "circ"), out))


def _check_equal(ref, got):
    np.testing.assert_allclose(got["ekei"], ref["ekei"], rtol=EKEI_RTOL, atol=0.0)
    for key in ("sfmin", "sfmax", "circ"):
        np.testing.assert_array_equal(got[key], ref[key])


@pytest.mark.gpu
@pytest.mark.parametrize("b,tdt", CASES, ids=IDS)
def test_noalloc_diag_matches_diag_twice(b, tdt):
    g = _stepped(b, tdt)
    ref = g.diag()
    for _ in range(2):
        rc, got = _call(g)
        assert rc == 0
        _check_equal(ref, got)
    # and after the state moves on
    g.step(tdt, 1)
    ref = g.diag()
    for _ in range(2):
        _check_equal(ref, g.diag_noalloc())
    g.close()


@pytest.mark.gpu
def test_noalloc_diag_mixed_precision():
    b = ocean_double_gyre(129, precision=OQG_MIXED)
    g = _stepped(b, 3600.0)
    ref = g.diag()
    for _ in range(2):
        _check_equal(ref, g.diag_noalloc())
    g.close()


@pytest.mark.gpu
def test_noalloc_diag_rejects_basin_over_the_scratch_limit():
    # 40 + 4 * nl * nyp doubles must fit in 32768: nl = 3, nyp = 2731 does not
    b = ocean_double_gyre(17)
    b.nyp = 2731
    g = QG(b)
    rc, got = _call(g)
    assert rc == 8                      # OQG_ESCRATCH
    assert np.all(np.isnan(got["ekei"]))  # nothing written
    with pytest.raises(OqgError):
        g.diag_noalloc()
    g.close()
