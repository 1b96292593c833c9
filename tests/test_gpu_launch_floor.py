"""The launch floor of the step chain (oqg_launch_floor): the step kernels'
launch shapes with no work, replayed from a graph, cost a small part of a
step; the measured step is well above it."""
import pytest

from openqg_b200.core import QG
from openqg_b200.params import double_gyre_tau, initial_psi, ocean_double_gyre
from openqg_b200.core import ekman_from_tau

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _need_gpu(gpu_required):
    pass


def test_launch_floor_is_a_small_part_of_a_step():
    b = ocean_double_gyre(513, dx=10e3)
    g = QG(b)
    p = b.fnot * initial_psi(b, 1)
    g.set_state(p, p)
    w, ts, tn = ekman_from_tau(b, *double_gyre_tau(b))
    g.set_forcing(w, None, ts, tn)
    assert g.step_launches() == 5
    floor = g.launch_floor(16)
    ms = g.profile_phases(3600.0, 5)
    assert 0.0 < floor < 0.5 * 1000.0 * sum(ms), (floor, ms)
    g.close()
