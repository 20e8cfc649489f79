"""The matching kernel's one device wait gives up with an error status.

A window's input arrives by a bulk copy whose completion the warp waits for
on an mbarrier, at most a bounded number of try_wait rounds; past that the
unit stops, the launch records a timeout and ngap_engine_sync returns
NGAP_E_TIMEOUT (the reference's kernels have no bounded waits: they poll
their worklists, code/src/ngap/kernel_ngap_OA.cu:142). The test hook
ngap_engine_test_wait_timeout leaves one unit's first copy unissued, so the
wait runs out with nothing in flight, and shortens the bound: no fault, no
hang, and the engine must match normally afterwards.
"""
import ctypes

import numpy as np
import pytest

import ngap_b200 as nb
from ngap_b200 import workloads as W
from ngap_b200._lib import lib
from oracle import oracle

NGAP_E_TIMEOUT = 8


@pytest.mark.gpu
@pytest.mark.parametrize("unit", [0, 3])
def test_wait_runs_out_then_engine_recovers(engine, unit):
    anml, data = W.hamming_set(seed=31, n_patterns=30, input_len=1 << 16, plant_every=1 << 11)
    groups = nb.Groups(nb.Nfa.from_string(anml), group_num=2)
    tables = nb.Tables(groups, precompute_depth=3)
    want, _ = oracle.match(groups.views(), data, 4, len(data) // 4)
    assert len(want) > 10
    got = engine.match(tables, data, 4, len(data) // 4, algorithm="nonblockingpcgroups")
    assert np.array_equal(got, want)

    assert lib().ngap_engine_test_wait_timeout(engine._h, unit, 1024) == 0
    engine.match_async(tables, data, 4, len(data) // 4, algorithm="nonblockingpcgroups")
    with pytest.raises(nb.NgapError) as ex:
        engine.sync()
    assert ex.value.status == NGAP_E_TIMEOUT
    assert "wait gave up" in str(ex.value)

    # the hook covered one match: the next ones run to completion
    for _ in range(2):
        got = engine.match(tables, data, 4, len(data) // 4, algorithm="nonblockingpcgroups")
        assert np.array_equal(got, want)


def test_hook_rejects_bad_arguments(built):
    assert lib().ngap_engine_test_wait_timeout(None, 0, 16) == 1
    assert lib().ngap_engine_test_wait_timeout(ctypes.c_void_p(0), -1, 16) == 1
