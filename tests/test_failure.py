"""Failure detection on the GPU without a fault: a resident CTA withholds its
first publish (test hook), so the other CTAs' bounded waits run out; the
launch ends early, the host reads FW_ERR_TIMEOUT at the next synchronising
call, and the context keeps working afterwards."""

import time

import pytest

import flatworld_b200 as fw
from flatworld_b200 import _native
from tests import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("res_sync", [0, 1], ids=["flag-in-data", "counter"])
def test_resident_wait_runs_out_and_the_context_recovers(res_sync):
    lp = fw.ExplicitLoop(0.0, scenes.plain_large_scene(fw, n=32, hf_offset=0.17), useAdapativeDT=True,
                         path="resident", patches=16, res_sync=res_sync)
    nw = lp._native
    assert lp.path == 2
    lp.advance_n(20)
    lp.synchronize()
    nw.set_option(_native.FW_OPT_WAIT_LIMIT, 4096)  # a few milliseconds of polling
    nw.set_option(_native.FW_OPT_TEST_WITHHOLD, 3)
    t0 = time.perf_counter()
    lp.advance_n(10)
    with pytest.raises(RuntimeError, match="gave up"):
        lp.synchronize()
    assert time.perf_counter() - t0 < 10.0
    nw.set_option(_native.FW_OPT_TEST_WITHHOLD, -1)
    lp.advance_n(10)
    lp.synchronize()  # the next launch clears the flag and runs to the end
    assert lp._native.read_counters(1)[0] > 0
    # (the state left by the aborted launch is not specified; only that the context works)
