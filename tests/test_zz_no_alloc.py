"""The entry point that allocates nothing: rsx_sim8_persistent_noalloc.

It exists for callers that cannot call cudaMalloc (their device memory belongs to another allocator, or an allocation
would synchronise a real-time loop): the persistent kernel's work-queue counter lives in a fixed 256-byte device array
of the library instead of a caller buffer.  This file runs last (pytest collects files by name), so a stop at the
first failure has run every other test before it.  It compares the entry point with rsx_sim8_persistent_raw, which
takes the counter from the caller, bit for bit (the decision is integer-exact: no tolerance) on two calls in a row, and
checks that a call beyond the array's limits is refused before anything launches."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_ARENAS = 1 << 24


def _bind(L):
    vp, u32 = ctypes.c_void_p, ctypes.c_uint32
    L.rsx_sim8_persistent_noalloc.argtypes = [vp, u32, vp, vp, vp, vp, vp, vp, u32, u32, u32, vp]
    L.rsx_sim8_persistent_noalloc.restype = ctypes.c_int
    return L.rsx_sim8_persistent_noalloc


def test_noalloc_matches_persistent_on_two_calls(rsx):
    import torch

    L = rsx.lib()
    noalloc = _bind(L)
    dev = rsx.SimDevice(0)
    try:
        sds = np.stack([rsx.build_static(7, p, q) for p, q in [(0, 0), (3, 1), (6, 4)]])
        n = 777  # not a multiple of 32: the last warp's lanes run past n
        idx = (np.arange(n) % 3).astype(np.uint8)
        st = rsx.make_states_multi(sds, idx, 11, rsx.MIX_CONTACT_HEAVY)
        dsd = dev.upload_static(sds)
        didx = torch.from_numpy(idx).to(dev.device)
        ref_states, new_states = dev.upload_states(st), dev.upload_states(st)
        ref_res, new_res = dev.alloc_result(n), dev.alloc_result(n)
        ref_ev = torch.zeros(n, dtype=torch.int32, device=dev.device)
        new_ev = torch.zeros(n, dtype=torch.int32, device=dev.device)
        counter = torch.zeros(1, dtype=torch.int32, device=dev.device)
        order = torch.from_numpy(np.random.default_rng(2).permutation(n).astype(np.int32)).to(dev.device)
        torch.cuda.synchronize()
        for call, (grid, gran, ordr) in enumerate([(148, 1, None), (37, 2, order)]):
            ctl = dev.upload_controls(rsx.decision_controls(5, call, n))
            op = ordr.data_ptr() if ordr is not None else None
            rsx.check(L.rsx_sim8_persistent_raw(ref_states.ptr(), n, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), ref_res.data_ptr(),
                                                ref_ev.data_ptr(), op, counter.data_ptr(), grid, 32, gran, dev.stream_ptr()),
                      "rsx_sim8_persistent_raw")
            rsx.check(noalloc(new_states.ptr(), n, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), new_res.data_ptr(), new_ev.data_ptr(), op,
                              grid, 32, gran, dev.stream_ptr()), "rsx_sim8_persistent_noalloc")
            dev.sync()
            want, got = dev.download_words(ref_states), dev.download_words(new_states)
            assert np.array_equal(want, got), f"call {call}: states differ"
            assert np.array_equal(ref_res.cpu().numpy(), new_res.cpu().numpy()), f"call {call}: results differ"
            assert np.array_equal(ref_ev.cpu().numpy(), new_ev.cpu().numpy()), f"call {call}: event words differ"
            assert not np.any(new_res.cpu().numpy().view(np.uint32) & (rsx.OVERFLOW | rsx.UNIMPLEMENTED))
        # more arenas than the fixed scratch allows: refused with a message, nothing launched
        rc = noalloc(new_states.ptr(), MAX_ARENAS + 1, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), new_res.data_ptr(), None, None, 148, 32, 1,
                     dev.stream_ptr())
        assert rc == -1
        assert b"16,777,216" in L.rsx_last_error()
        # granularity past 256, grid past 65,535, a block that is not 32 or 64: refused the same way
        for grid, block, gran in ((148, 32, 257), (65536, 32, 1), (148, 96, 1)):
            rc = noalloc(new_states.ptr(), n, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), new_res.data_ptr(), None, None, grid, block, gran,
                         dev.stream_ptr())
            assert rc == -1, (grid, block, gran)
        dev.sync()
        assert np.array_equal(dev.download_words(new_states), got)
        for h in (ref_states, new_states, dsd):
            h.free()
    finally:
        dev.close()
