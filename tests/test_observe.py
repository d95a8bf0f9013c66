"""Observations and rewards (rsx_observe_raw, k_observe) against the NumPy restatement in oracle/observe.py, bit for
bit: FP16 observation rows and FP32 rewards of both cars of every arena, after decisions with contacts, goals and
pickups, over several car pairings and an arena count that is not a multiple of 32."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import observe as OB  # noqa: E402


def test_pad_mirror_matches_oracle(rsx):
    sds = np.stack([rsx.build_static(7, p, q) for p, q in [(0, 0), (3, 5)]])
    got = rsx.pad_mirror(sds)
    for k in range(sds.shape[0]):
        assert np.array_equal(got[k], OB.pad_mirror(sds[k]))
    m = got[0].astype(int)
    assert np.array_equal(m[m], np.arange(34)), "mirroring twice gives the pad back"


def test_oracle_layout_by_hand(rsx):
    sd = rsx.build_static(7, 0, 0)
    st = rsx.make_states(sd, 3, 4, rsx.MIX_HEADLINE)
    obs, rew = OB.observe(st, sd[None], None, rsx.pad_mirror(sd), None, None, np.zeros(8, np.float32))
    f = st.view(np.float32)
    ball = OB._w(OB.A["ball"][0])
    want = (f[:, ball:ball + 3] * OB.POS).astype(np.float16).view(np.uint16)
    assert np.array_equal(obs[0::2, 0:3], want)
    flip = (f[:, ball:ball + 3] * np.array([-1, -1, 1], np.float32) * OB.POS).astype(np.float16).view(np.uint16)
    assert np.array_equal(obs[1::2, 0:3], flip)
    assert np.all(obs[:, 102:] == 0) and np.all(rew == 0)


@pytest.mark.gpu
def test_observe_kernel_matches_oracle(rsx):
    import torch

    from runner import DecisionRunner

    n = 4099
    sds = np.stack([rsx.build_static(7, p, q) for p, q in [(0, 0), (2, 3), (6, 5)]])
    idx = (np.arange(n) * 7 % 3).astype(np.uint8)
    st = rsx.make_states_multi(sds, idx, 11, rsx.MIX_CONTACT_HEAVY)
    dev = rsx.SimDevice(0)
    try:
        run = DecisionRunner(dev, sds, idx, st)
        weights = np.array([10.0, 0.5, 0.25, 2.0, -2.0, 0.125, 0.01, 0.02], np.float32)
        seen = {"scored": 0, "touch": 0, "pickup": 0}
        for d in range(3):
            ctl = torch.from_numpy(rsx.decision_controls(77, d, n).view(np.int32)).to(dev.device)
            run.step(ctl.data_ptr(), {"mode": "lockstep", "block": 448, "grid": run.sms, "split": 7, "threshold": None})
            obs, rew = run.observe(weights)
            run.stream.synchronize()
            states = dev.download_states(run.ds)
            res = run.res.cpu().numpy().view(np.uint32)
            ev = run.ev.cpu().numpy().view(np.uint32)
            want_obs, want_rew = OB.observe(states, sds, idx, rsx.pad_mirror(sds), res, ev, weights)
            got_obs = obs.cpu().numpy().view(np.uint16)
            got_rew = rew.cpu().numpy()
            bad = np.nonzero(np.any(got_obs != want_obs, axis=1))[0]
            assert bad.size == 0, f"decision {d}: rows {bad[:8]}, columns {np.nonzero(got_obs[bad[0]] != want_obs[bad[0]])[0]}"
            assert np.array_equal(got_rew.view(np.uint32), want_rew.view(np.uint32)), f"decision {d}: rewards"
            seen["scored"] += int(((res & 0xFF) != 0).sum())
            seen["touch"] += int(((ev & 3) != 0).sum())
            seen["pickup"] += int((((ev >> 6) & 3) != 0).sum())
        assert seen["touch"] > 0 and seen["pickup"] > 0, seen
        run.free()
    finally:
        dev.close()
