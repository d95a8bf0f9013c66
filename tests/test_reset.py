"""Device resets (rsx_reset_arenas_raw): the fresh start states the device writes equal the host generator's word for
word (same seed, arena index, car pairing and scenario mix), and only the selected arenas change."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_device_reset_matches_host_states_and_selection(rsx):
    import torch

    n = 777
    sds = np.stack([rsx.build_static(7, p, q) for p, q in [(0, 0), (3, 5), (6, 1)]])
    idx = (np.arange(n) * 7 % 3).astype(np.uint8)
    mix = (ctypes.c_float * 5)(*rsx.MIX_HEADLINE)
    dev = rsx.SimDevice(0)
    try:
        L = rsx.lib()
        dsd = dev.upload_static(sds)
        didx = torch.from_numpy(idx).to(dev.device)
        count = torch.zeros(1, dtype=torch.int32, device=dev.device)
        # every arena, over a buffer of other states: the host's states for seed 42
        old = rsx.make_states_multi(sds, idx, 9, rsx.MIX_CONTACT_HEAVY)
        ds = dev.upload_states(old)
        rsx.check(L.rsx_reset_arenas_raw(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), 42, mix, None, None, count.data_ptr(), dev.stream_ptr()),
                  "reset")
        dev.sync()
        want = rsx.make_states_multi(sds, idx, 42, rsx.MIX_HEADLINE)
        got = dev.download_states(ds)
        assert np.array_equal(got, want)
        assert int(count.item()) == n
        # a mask and "scored" result words: only arenas with both change
        ds2 = dev.upload_states(old)
        mask = (np.arange(n) % 3 == 0).astype(np.uint8)
        result = np.where(np.arange(n) % 2 == 0, 5, 0).astype(np.uint32)
        result[7] |= 0x80000000  # flags do not count as a goal; arena 7 (not a multiple of 2) stays
        dm = torch.from_numpy(mask).to(dev.device)
        dr = torch.from_numpy(result.view(np.int32)).to(dev.device)
        count.zero_()
        torch.cuda.synchronize()
        rsx.check(L.rsx_reset_arenas_raw(ds2.ptr(), n, dsd.ptr(), didx.data_ptr(), 42, mix, dr.data_ptr(), dm.data_ptr(), count.data_ptr(),
                                         dev.stream_ptr()), "reset")
        dev.sync()
        got2 = dev.download_states(ds2)
        sel = (mask != 0) & ((result & 0xFF) != 0)
        assert np.array_equal(got2[sel], want[sel])
        assert np.array_equal(got2[~sel], old[~sel])
        assert int(count.item()) == int(sel.sum())
        ds.free()
        ds2.free()
        dsd.free()
    finally:
        dev.close()
