"""The bounded device-wait path: a wait that nothing completes gives up,
reports VEXT_ERR_TIMEOUT (17) with a message, and leaves the device usable.

Every staged pair kernel waits on mbarriers for its bulk copies; those waits
are bounded so that a copy that never lands becomes a status the host
reports instead of a hung GPU.  ``vext_check_wait_timeout`` runs that same
bounded wait on a barrier armed for a copy that is never issued (nothing in
flight), with a short poll limit passed at run time."""
import numpy as np
import pytest

from oracle import oracle
from string_vext_b200 import _lib, synth
from string_vext_b200.orientation import normalized_directors, regular_pose_grid
from string_vext_b200.system import VextSystem

pytestmark = pytest.mark.gpu


def test_wait_gives_up_with_status_17_and_device_stays_usable():
    lib = _lib.load()
    assert lib.vext_check_wait_timeout(1024) == _lib.VEXT_ERR_TIMEOUT
    assert b"gave up after 1024 polls" in lib.vext_last_error()
    # a regular field call on the same device right after: status 0, right values
    case = synth.small_field()
    centers, axes = regular_pose_grid(3, 64)
    axes = normalized_directors(axes)
    with VextSystem(case) as system:
        e = system.field(3, axes, mode=_lib.VEXT_MODE_FP64, energy=True)["energy"]
    ref = oracle.pose_energy(case, centers, axes)
    assert (np.abs(e - ref) / np.maximum(np.abs(ref), 1.0)).max() < 1e-10
    assert lib.vext_check_wait_timeout(1) == _lib.VEXT_ERR_TIMEOUT


@pytest.mark.parametrize("polls", [0, -5, (1 << 22) + 1])
def test_wait_limit_out_of_range_is_an_argument_error(polls):
    lib = _lib.load()
    assert lib.vext_check_wait_timeout(polls) == _lib.VEXT_ERR_ARGUMENT
