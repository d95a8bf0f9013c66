"""What the trained contact predictor gains: the lockstep kernel over the identity order, over an untrained network's
order and over the trained network's orders (two bins, sixteen cost levels), 262,144 arenas of the headline mix
(several claim rounds per SM, where the order matters), timed on the same decisions from the same start states.  The
test checks what must hold — every order gives the same words, and the trained network's recall and precision on
these decisions — and prints the timings (run with -s to see them); the speed-ups are measurements, not pass
conditions.  With the lockstep kernel's pooled contact work (splits 9 to 15) the heavy arenas' leaf tests are spread over
the block, and the orders measure within a few percent of the identity order either way (best of three, 262,144 and
1,048,576 arenas after 8 decisions: two bins +0.7% / +2.2%, sixteen levels -1.5% / +0.8%), inside the spread of
repeated runs, so no gain is asserted."""
import json
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trained_order_gain_is_measured_and_exact(rsx):
    import torch

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import predictor as P
    from runner import DecisionRunner

    n = 262144
    dev = rsx.SimDevice(0)
    try:
        sds, idx, st = bench.world(rsx, n, 0, 3)
        run = DecisionRunner(dev, sds, idx, st)
        D = 3
        ctl = [torch.from_numpy(rsx.decision_controls(4242, d, n).view(np.int32)).to(dev.device) for d in range(D)]
        torch.cuda.synchronize()
        start = run.snapshot()
        run.pred = P.ContactPredictor(dev.device, seed=3, stream=run.sptr)  # untrained weights

        def timed(cfg):
            run.restore(start)
            run.stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(run.stream)
            for c in ctl:
                run.step(c.data_ptr(), cfg)
            e1.record(run.stream)
            e1.synchronize()
            return e0.elapsed_time(e1), run.snapshot().cpu().numpy(), run.res.cpu().numpy().copy()

        base = {"block": 448, "grid": run.sms, "split": 15}
        for_warm = timed({"mode": "lockstep", **base})  # first launches load the kernels
        t_id, w_id, r_id = timed({"mode": "lockstep", **base})
        t_un, w_un, r_un = timed({"mode": "binned", "threshold": 0.5, **base})
        run.pred = None
        run.train_predictor(control_seed=777, decisions=8)
        t_tr, w_tr, r_tr = timed({"mode": "binned", "threshold": 0.5, **base})
        t_lv, w_lv, r_lv = timed({"mode": "levels", "levels": 16, "weights": [1.0] * 6, **base})
        assert np.array_equal(w_id, w_un) and np.array_equal(w_id, w_tr) and np.array_equal(w_id, for_warm[1]) and np.array_equal(w_id, w_lv)
        assert np.array_equal(r_id, r_un) and np.array_equal(r_id, r_tr) and np.array_equal(r_id, r_lv)
        # recall / precision of the trained network on these decisions
        run.restore(start)
        Zs, Ys = [], []
        with torch.cuda.stream(run.stream):
            for c in ctl:
                run.step(c.data_ptr(), {"mode": "binned", "threshold": 0.5, **base})
                Zs.append(run.Z.clone())
                Ys.append(run.pred.labels(run.ev.data_ptr(), n).clone())
        run.stream.synchronize()
        m = P.recall_precision(torch.cat(Zs).cpu().numpy(), torch.cat(Ys).cpu().numpy())
        assert m["any"][0] > 0.8 and m["any"][1] > 0.8, m["any"]
        print(json.dumps({"arenas": n, "decisions": D, "ms_identity_order": round(t_id, 2), "ms_untrained_order": round(t_un, 2),
                          "ms_trained_order": round(t_tr, 2), "ms_trained_levels": round(t_lv, 2), "gain_vs_identity": round(t_id / t_tr, 4),
                          "levels_gain_vs_identity": round(t_id / t_lv, 4),
                          "gain_vs_untrained": round(t_un / t_tr, 4), "any_contact_recall_precision": [round(float(x), 3) for x in m["any"][:2]]}))
        run.free()
    finally:
        dev.close()
