"""The bounded device waits give up, flag and return (no hung GPU).

Each probe runs the library's own wait function (grid barrier, ordered-append
look-back, mbarrier wait) on a wait nothing can satisfy, with a limit of a
thousand polls instead of the kernels' 2^20.  The probe must end by itself
with MK_DEVICE_WAIT_TIMEOUT_FLAG raised and every launched block finished,
and the GPU must stay usable: a tick run afterwards matches the oracle bit
for bit.
"""
import pytest

from mechanic_b200 import abi, scenes
from mechanic_b200.physics import selftest_bounded_wait

from test_gpu_parity import compare_tick, make_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", [abi.WAIT_PROBE_GRID_BARRIER, abi.WAIT_PROBE_LOOKBACK, abi.WAIT_PROBE_MBARRIER],
                         ids=["grid-barrier", "lookback", "mbarrier"])
def test_wait_gives_up_flags_and_returns(cuda_lib, which):
    r = selftest_bounded_wait(which, spin_limit=1000)
    assert r.error_flags & abi.DEVICE_WAIT_TIMEOUT_FLAG
    assert r.blocks_finished == r.blocks_launched >= 1
    assert r.elapsed_ms < 2000.0
    if which == abi.WAIT_PROBE_LOOKBACK:
        assert r.lookback_prefix == 0   # the missing predecessor counts as zero
    # the context is intact: a tick right after matches the oracle
    gpu, orc = make_pair(scenes.falling_cubes(200, seed=4))
    compare_tick(gpu, orc, 1)
    gpu.close()


def test_wait_probe_rejects_bad_arguments(cuda_lib):
    from mechanic_b200.physics import InvalidArgument
    with pytest.raises(InvalidArgument):
        selftest_bounded_wait(7, 1000)
    with pytest.raises(InvalidArgument):
        selftest_bounded_wait(abi.WAIT_PROBE_LOOKBACK, 0)
