"""The reference's own GPU kernel beside this project's, word for word.

oracle/_ref/sim8_ref.cubin is the reference's cuda/sim/sim.cu compiled unchanged for sm_100a (oracle/Makefile `gpu`).
Its sim8 and this project's reference-shaped entry rsx_sim8 (k_sim8) step the same AoSoA-32 buffers of the same start
states with the same controls; every tick-boundary word and every result word must be equal.  (The reference documents
its GPU build as bit-identical to its correctly rounded CPU build; the oracle tests pin this project's kernels to that
CPU build; this test ties the two GPU paths together directly.)"""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refsim():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refgpu

    if not refgpu.available():
        pytest.skip("oracle/_ref/sim8_ref.cubin not built")
    r = refgpu.RefSim8(0)
    yield r
    r.close()


@pytest.mark.parametrize("presets,mix", [((0, 0), "headline"), ((3, 5), "contact")])
def test_reference_sim8_equals_ours(rsx, refsim, presets, mix):
    import torch

    sd = rsx.build_static(7, *presets)
    n = 1000
    st = rsx.make_states(sd, n, 21, rsx.MIX_HEADLINE if mix == "headline" else rsx.MIX_CONTACT_HEAVY)
    dev = rsx.SimDevice(0)
    try:
        dsd = dev.upload_static(sd)
        ours = dev.upload_states(st)
        theirs = torch.from_numpy(rsx.pack(st).view(np.int32)).to(dev.device)
        res_o = dev.alloc_result(n)
        res_t = torch.zeros(n, dtype=torch.int32, device=dev.device)
        for d in range(4):
            ctl = dev.upload_controls(rsx.decision_controls(31, d, n))
            dev.sim8(ours, dsd, ctl, res_o)
            dev.sync()
            refsim.sim8(theirs.data_ptr(), n, dsd.ptr(), ctl.data_ptr(), res_t.data_ptr(), dev.stream_ptr())
            dev.sync()
            got = rsx.unpack(theirs.cpu().numpy().view(np.uint32), n)
            want = dev.download_states(ours)
            bad = np.nonzero(np.any(got[:, :rsx.TICK_WORDS] != want[:, :rsx.TICK_WORDS], axis=1))[0]
            assert bad.size == 0, f"decision {d}: arenas {bad[:8]} differ between the reference's sim8 and k_sim8"
            assert np.array_equal(res_t.cpu().numpy(), res_o.cpu().numpy()), f"decision {d}: result words differ"
        ours.free()
        dsd.free()
    finally:
        dev.close()
