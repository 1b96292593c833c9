"""Compensated summation of the mass-constraint and area integrals.

int_P_dA (numerics.F90:165-204) on the device sums with a running
compensation (TwoSum), so a field whose terms cancel to ten orders of
magnitude still integrates to within a few roundings of the exact sum of its
FP64 values (math.fsum), where a running FP64 sum of the same terms is off
by more than 1e-9 of the result.  The step's modal area integrals (box_homog) and
the entrainment integral use the same accumulation.
"""
import math

import numpy as np
import pytest

from openqg_b200.core import QG
from openqg_b200.params import OQG_MIXED, ocean_double_gyre

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu(gpu_required):
    pass


def _cancelling_field(b, seed, big=1.0e10):
    """big * (a pattern whose trapezoid integral is exactly zero: values
    mirrored with opposite signs about the centre column) + a smooth field
    of order one."""
    rng = np.random.default_rng(seed)
    r = rng.standard_normal(b.shape2)
    pat = r - r[:, ::-1]                     # antisymmetric in x: exact zero sum
    yy, xx = np.meshgrid(np.linspace(0, 1, b.nyp), np.linspace(0, 1, b.nxp), indexing="ij")
    smooth = 1.0 + np.cos(np.pi * xx) * np.sin(np.pi * yy)
    return big * pat + smooth


def _exact_int(b, f):
    w = np.ones(b.shape2)
    w[0, :] *= 0.5
    w[-1, :] *= 0.5
    w[:, 0] *= 0.5
    w[:, -1] *= 0.5
    return math.fsum((w * f).ravel().tolist()) * b.dx * b.dy


@pytest.mark.parametrize("n,prec", [(129, 0), (513, 0), (513, OQG_MIXED)])
def test_area_integral_is_compensated(n, prec):
    b = ocean_double_gyre(n, precision=prec)
    g = QG(b)
    for seed in (1, 2):
        f = _cancelling_field(b, seed)
        exact = _exact_int(b, f)
        got = g.int_P_dA(f)
        assert abs(got - exact) <= 1e-15 * abs(exact), (got, exact)
        # the same terms added one after another in FP64 (a running sum, as
        # an uncompensated loop forms it) miss by far more
        w = np.ones(b.shape2)
        w[[0, -1], :] *= 0.5
        w[:, [0, -1]] *= 0.5
        plain = float(np.cumsum((w * f).ravel(), dtype=np.float64)[-1]) * b.dx * b.dy
        assert abs(plain - exact) > 1e-9 * abs(exact)
    g.close()
