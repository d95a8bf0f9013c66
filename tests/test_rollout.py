"""An on-device rollout (rollout.Rollout): binned decisions with the predictor retrained online every 16 decisions and
goal-ended episodes restarted on the device, checked word for word on a 1% sample of its arenas against the oracle
replaying the same decisions (same controls, same restarts from the host generator) at decisions 1, 20 and 40."""
import os

import numpy as np
import pytest

from conftest import ORACLE_SO, Oracle

pytestmark = pytest.mark.gpu


def test_rollout_with_retraining_and_resets_matches_oracle(rsx):
    import torch

    import rollout
    from runner import DecisionRunner

    if not os.path.exists(ORACLE_SO):
        pytest.skip("needs the oracle library")
    orc = Oracle()
    n, D, K = 32768, 40, 4
    mix = rsx.MIX_CONTACT_HEAVY
    sds = np.stack([rsx.build_static(7, p, q) for p, q in [(0, 0), (2, 3), (6, 5)]])
    idx = (np.arange(n) * 5 % 3).astype(np.uint8)
    st = rsx.make_states_multi(sds, idx, 5, mix)
    dev = rsx.SimDevice(0)
    try:
        run = DecisionRunner(dev, sds, idx, st)
        host_pool = [rsx.decision_controls(31, k, n) for k in range(K)]
        pool = [torch.from_numpy(c.view(np.int32)).to(dev.device) for c in host_pool]
        run.train_predictor(control_seed=55, decisions=4, epochs=2)
        sample = np.sort(np.random.default_rng(8).choice(n, n // 100, replace=False))
        checks = {1, 20, 40}
        got = {}

        def on_decision(d):
            if d + 1 in checks:
                got[d + 1] = dev.download_states(run.ds)[sample]

        cfg = {"mode": "binned", "block": 448, "grid": run.sms, "split": 15, "threshold": 0.5}
        ro = rollout.Rollout(run, pool, reset_seed=99, mix=mix, config=cfg, sample_per_decision=8192)
        windows = ro.run_decisions(D, retrain_every=16, on_decision=on_decision)
        assert len(windows) == 3 and windows[-1]["decisions"] == [32, 39]
        assert all(w["overflow"] == 0 and w["unimplemented"] == 0 for w in windows)
        # the oracle's replay of the sample
        ref = st[sample].copy()
        resets = 0
        for d in range(D):
            ctl = host_pool[d % K][sample]
            scored = np.array([orc.decide(ref[j], sds[idx[sample[j]]], ctl[j]) for j in range(sample.size)])
            hit = np.nonzero(scored)[0]
            if hit.size:
                resets += hit.size
                ref[hit] = rsx.make_states_at(sds, idx[sample[hit]], sample[hit], 99 + d, mix)
            if d + 1 in checks:
                bad = np.nonzero(np.any(got[d + 1][:, :rsx.TICK_WORDS] != ref[:, :rsx.TICK_WORDS], axis=1))[0]
                assert bad.size == 0, f"decision {d + 1}: sampled arenas {sample[bad][:8]} differ from the oracle"
        assert resets > 0, "no episode ended in the sample: the restarts were not exercised"
        run.free()
    finally:
        dev.close()


def test_long_levels_rollout_matches_oracle_on_a_sample(rsx):
    """131,072 arenas x 60 decisions with the learned 16-level order (several claim rounds, so the order is far from the
    identity), retrained every 20 decisions, goal-ended episodes restarted on the device: a 0.2% sample checked word for
    word against the oracle at decisions 1, 30 and 60."""
    import torch

    import rollout
    from runner import DecisionRunner

    if not os.path.exists(ORACLE_SO):
        pytest.skip("needs the oracle library")
    orc = Oracle()
    n, D, K = 131072, 60, 6
    mix = rsx.MIX_HEADLINE
    sds = np.stack([rsx.build_static(7, p, q) for p, q in [(0, 0), (1, 4), (5, 2), (6, 6)]])
    idx = (np.arange(n) * 7 % 4).astype(np.uint8)
    st = rsx.make_states_multi(sds, idx, 21, mix)
    dev = rsx.SimDevice(0)
    try:
        run = DecisionRunner(dev, sds, idx, st)
        host_pool = [rsx.decision_controls(77, k, n) for k in range(K)]
        pool = [torch.from_numpy(c.view(np.int32)).to(dev.device) for c in host_pool]
        run.train_predictor(control_seed=56, decisions=4, epochs=2)
        sample = np.sort(np.random.default_rng(3).choice(n, n // 500, replace=False))
        checks = {1, 30, 60}
        got = {}

        def on_decision(d):
            if d + 1 in checks:
                got[d + 1] = dev.download_states(run.ds)[sample]

        cfg = {"mode": "levels", "block": 448, "grid": run.sms, "split": 15, "threshold": None, "levels": 16, "weights": [1.0] * 6}
        ro = rollout.Rollout(run, pool, reset_seed=123, mix=mix, config=cfg, sample_per_decision=8192)
        windows = ro.run_decisions(D, retrain_every=20, on_decision=on_decision)
        assert len(windows) == 3 and all(w["overflow"] == 0 and w["unimplemented"] == 0 for w in windows)
        ref = st[sample].copy()
        resets = 0
        for d in range(D):
            ctl = host_pool[d % K][sample]
            scored = np.array([orc.decide(ref[j], sds[idx[sample[j]]], ctl[j]) for j in range(sample.size)])
            hit = np.nonzero(scored)[0]
            if hit.size:
                resets += hit.size
                ref[hit] = rsx.make_states_at(sds, idx[sample[hit]], sample[hit], 123 + d, mix)
            if d + 1 in checks:
                bad = np.nonzero(np.any(got[d + 1][:, :rsx.TICK_WORDS] != ref[:, :rsx.TICK_WORDS], axis=1))[0]
                assert bad.size == 0, f"decision {d + 1}: sampled arenas {sample[bad][:8]} differ from the oracle"
        assert resets > 0, "no episode ended in the sample: the restarts were not exercised"
        run.free()
    finally:
        dev.close()
