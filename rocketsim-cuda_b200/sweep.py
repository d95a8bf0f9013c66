"""Arena-count sweep of the decision step: the plain launch, the lockstep kernel and the lockstep kernel with the learned
binning (two bins, and sixteen cost levels), at 4,096 ... 1,048,576 arenas of one workload, each timed on the same decisions from the same start states,
with the runs' words compared (all arenas, on the device).  One JSON line per size.

  python rocketsim-cuda_b200/sweep.py [--sizes 4096,16384,65536,262144,1048576] [--decisions 4] [--mix headline]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="4096,16384,65536,262144,1048576")
    ap.add_argument("--decisions", type=int, default=4)
    ap.add_argument("--mix", default="headline", choices=["headline", "contact"])
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args()
    import torch

    import bench
    import rsx
    from runner import DecisionRunner

    mix = rsx.MIX_HEADLINE if args.mix == "headline" else rsx.MIX_CONTACT_HEAVY
    dev = rsx.SimDevice(0)
    sds = np.stack([rsx.build_static(7, p, q) for p, q in bench.PRESETS])
    for n in [int(x) for x in args.sizes.split(",")]:
        with np.errstate(over="ignore"):
            h = rsx._mix64(np.arange(n, dtype=np.uint64) + np.uint64(1 << 40))
        idx = (h % np.uint64(len(bench.PRESETS))).astype(np.uint8)
        st = rsx.make_states_multi(sds, idx, args.seed, mix)
        run = DecisionRunner(dev, sds, idx, st)
        del st
        ctl = [torch.from_numpy(rsx.decision_controls(args.seed * 1000, d, n).view(np.int32)).to(dev.device) for d in range(args.decisions + 1)]
        torch.cuda.synchronize()
        start = run.snapshot()
        t0 = time.perf_counter()
        run.train_predictor(control_seed=args.seed * 1000 + 500, decisions=max(2, 2097152 // n))
        train_s = time.perf_counter() - t0
        base = {"block": 448, "grid": run.sms, "split": 7}
        out, words = {}, {}
        for name, cfg in [("plain", {"mode": "plain", "block": 32}), ("lockstep", {"mode": "lockstep", **base}),
                          ("binned", {"mode": "binned", "threshold": 0.5, **base}),
                          ("levels", {"mode": "levels", "levels": 16, "weights": [1.0] * 6, **base})]:
            run.restore(start)
            run.step(ctl[0].data_ptr(), cfg)  # the first launch of a kernel loads it: outside the timing
            run.stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(run.stream)
            for d in range(1, args.decisions + 1):
                run.step(ctl[d].data_ptr(), cfg)
            e1.record(run.stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / args.decisions
            out[name] = {"ms_per_decision": round(ms, 3), "arena_ticks_per_s": n * 8 / (ms / 1e3)}
            words[name] = (run.snapshot(), run.res.clone())
        exact = all(torch.equal(words[k][0], words["plain"][0]) and torch.equal(words[k][1], words["plain"][1]) for k in words)
        print(json.dumps({"arenas": n, "mix": args.mix, "decisions": args.decisions, "train_s": round(train_s, 2), **out,
                          "lockstep_vs_plain": out["plain"]["ms_per_decision"] / out["lockstep"]["ms_per_decision"],
                          "binned_vs_plain": out["plain"]["ms_per_decision"] / out["binned"]["ms_per_decision"],
                          "levels_vs_plain": out["plain"]["ms_per_decision"] / out["levels"]["ms_per_decision"],
                          "bit_exact_all_arenas": bool(exact)}), flush=True)
        del words, start
        run.free()
        del run
        torch.cuda.empty_cache()


if __name__ == "__main__":
    main()
