"""The bench's word-for-word check against the oracle, on the CPU.

rsref_run_batch_ex (oracle/batch.cpp) runs the reference's CPU build over many arenas and reports each decision's result
word and event OR as the decision kernels write them; bench.oracle_compare replays a sample of a workload through it and
counts mismatches.  Here both are checked without a GPU: the batch driver against arena-by-arena calls of the oracle
with its per-tick trace (the bookkeeping: control rows through an index map, event OR up to the goal, the overflow and
unimplemented bits), and the comparison against this project's host build of the same decisions (rsx_host_decide),
which must report no mismatch, and one planted change in each kind of word, which it must report."""
import ctypes
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

BATCH_SO = os.path.join(ROOT, "oracle", "_ref", "librsbatch.so")
EVENTS_WORD = 2566


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


@pytest.fixture(scope="module")
def bench():
    if not os.path.exists(BATCH_SO):
        pytest.skip("oracle/_ref not built")
    sys.path.insert(0, ROOT)
    import bench as B

    return B


def test_batch_ex_matches_arena_by_arena_oracle(rsx, oracle, bench):
    L = bench.oracle_batch()
    sds = np.stack([rsx.build_static(7, p, q) for p, q in [(0, 0), (2, 5)]])
    n, decisions = 40, 3
    idx = (np.arange(n) % 2).astype(np.uint8)
    st = rsx.make_states_multi(sds, idx, 4, rsx.MIX_CONTACT_HEAVY)
    ctl = bench.controls_of(rsx, 9, 0, decisions, 100)  # rows of a 100-arena workload; the sample reads rows 7, 9, ...
    rows = (7 + 2 * np.arange(n)).astype(np.uint32)
    got = st.copy()
    res = np.zeros((decisions, n), np.uint32)
    ev = np.zeros((decisions, n), np.uint32)
    L.rsref_run_batch_ex(got.ctypes.data, n, sds.ctypes.data, idx.ctypes.data, ctl.ctypes.data, 100, rows.ctypes.data, decisions, 3,
                         res.ctypes.data, ev.ctypes.data)
    want = st.copy()
    for a in range(n):
        for d in range(decisions):
            trace = np.zeros((8, rsx.ARENA_WORDS), np.uint32)
            sc = ctypes.c_uint32(0)
            status = oracle.L.rscuda_step_ticks(_p(want[a]), _p(sds[idx[a]]), _p(np.ascontiguousarray(ctl[d, rows[a]])), 8, ctypes.byref(sc),
                                                _p(trace))
            upto = sc.value or 8
            e = int(np.bitwise_or.reduce(trace[:upto, EVENTS_WORD]))
            r = sc.value | (0x80000000 if status != 0 else 0) | (0x40000000 if np.any(want[a, 2560:2566]) else 0)
            assert res[d, a] == r and ev[d, a] == e, (a, d)
    assert np.array_equal(got, want)
    assert np.any(ev != 0)


def test_oracle_compare_agrees_with_host_build_and_reports_changes(rsx, bench):
    """The host build of this project's simulator (the same source as the kernels) stands in for the GPU: no mismatch;
    a flipped state word, result word or event word in the compared data: reported."""
    L = bench.oracle_batch()
    H = rsx.lib()
    sds = np.stack([rsx.build_static(7, p, q) for p, q in [(1, 1), (6, 3)]])
    n, decisions = 24, 2
    idx = (np.arange(n) % 2).astype(np.uint8)
    st = rsx.make_states_multi(sds, idx, 6, rsx.MIX_HEADLINE)
    ctl = bench.controls_of(rsx, 12, 0, decisions, n)
    cur = st.copy()
    res = np.zeros((decisions, n), np.uint32)
    for d in range(decisions):
        for a in range(n):
            res[d, a] = H.rsx_host_decide(_p(cur[a]), _p(sds[idx[a]]), _p(np.ascontiguousarray(ctl[d, a])))
    sample = np.arange(n)
    # the event OR is not returned by the host decide: take the oracle's own and check the states and result words
    ev_ref = np.zeros((decisions, n), np.uint32)
    res_ref = np.zeros((decisions, n), np.uint32)
    tmp = st.copy()
    L.rsref_run_batch_ex(tmp.ctypes.data, n, sds.ctypes.data, idx.ctypes.data, ctl.ctypes.data, n, None, decisions, 2, res_ref.ctypes.data,
                         ev_ref.ctypes.data)
    assert np.array_equal(res, res_ref)
    m = bench.oracle_compare(L, sds, idx, st, ctl, sample, cur, res, ev_ref)
    assert m["mismatches"] == 0 and m["arenas"] == n and m["decisions"] == decisions
    bad = cur.copy()
    bad[5, 100] ^= 1
    assert bench.oracle_compare(L, sds, idx, st, ctl, sample, bad, res, ev_ref)["state_mismatches"] == 1
    r2 = res.copy()
    r2[1, 7] ^= 0x40000000
    assert bench.oracle_compare(L, sds, idx, st, ctl, sample, cur, r2, ev_ref)["result_mismatches"] == 1
    e2 = ev_ref.copy()
    e2[0, 3] ^= 4
    m = bench.oracle_compare(L, sds, idx, st, ctl, sample, cur, res, e2)
    assert m["event_mismatches"] == 1 and m["first_bad"] == [3]
