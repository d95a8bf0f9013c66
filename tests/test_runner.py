"""The batching layer (runner.DecisionRunner): the plain launch, the lockstep kernel launched one by one and as a CUDA
graph, and the learned-binning order give the same words after several decisions, and the autotuner leaves the states
as it found them (it times candidates on a snapshot)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_modes_graphs_and_autotuner_agree(rsx):
    import torch
    from runner import DecisionRunner

    n = 2000
    sds = np.stack([rsx.build_static(7, p, q) for p, q in [(0, 0), (1, 4), (6, 6)]])
    idx = (np.arange(n) % 3).astype(np.uint8)
    st = rsx.make_states_multi(sds, idx, 9, rsx.MIX_CONTACT_HEAVY)
    dev = rsx.SimDevice(0)
    try:
        run = DecisionRunner(dev, sds, idx, st)
        D = 4
        ctl = [torch.from_numpy(rsx.decision_controls(21, d, n).view(np.int32)).to(dev.device) for d in range(D)]
        torch.cuda.synchronize()
        start = run.snapshot()
        run.train_predictor(control_seed=77, decisions=2, epochs=1)
        modes = [{"mode": "plain", "block": 32},
                   {"mode": "lockstep", "block": 448, "grid": run.sms, "split": 1},
                   {"mode": "lockstep", "block": 64, "grid": 3, "split": 0},
                   {"mode": "binned", "block": 384, "grid": run.sms, "split": 1, "threshold": 0.3}]
        outs = []
        for i, c in enumerate(modes):
            run.restore(start)
            # the last mode runs with the static data in a persisting L2 window (a cache hint: same words)
            if i == len(modes) - 1:
                rsx.check(rsx.lib().rsx_l2_persist_raw(run.dsd.ptr(), sds.size * 4, 1.0, run.sptr), "l2 window")
            if i == 1:  # as one CUDA graph of all D decisions
                g = run.capture([x.data_ptr() for x in ctl], c)
                run.replay(g)
            else:
                for x in ctl:
                    run.step(x.data_ptr(), c)
            run.stream.synchronize()
            outs.append((run.snapshot().cpu().numpy(), run.res.cpu().numpy().copy(), run.ev.cpu().numpy().copy()))
        for i, o in enumerate(outs[1:], 1):
            assert np.array_equal(o[0], outs[0][0]), f"{modes[i]}: states differ"
            assert np.array_equal(o[1], outs[0][1]), f"{modes[i]}: results differ"
            assert np.array_equal(o[2], outs[0][2]), f"{modes[i]}: event words differ"
        rsx.check(rsx.lib().rsx_l2_persist_raw(None, 0, 0.0, run.sptr), "l2 window off")
        # the autotuner times on a snapshot and restores it
        run.restore(start)
        before = run.snapshot().cpu().numpy()
        res = run.tune([x.data_ptr() for x in ctl[:1]], run.candidates()[:4])
        assert len(res) == 4 and res[0][0] <= res[-1][0]
        run.stream.synchronize()
        assert np.array_equal(run.snapshot().cpu().numpy(), before)
        run.free()
    finally:
        dev.close()
