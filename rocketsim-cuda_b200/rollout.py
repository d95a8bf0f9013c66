"""On-device rollouts: many decisions of one batch of arenas, with the learned binning retrained online from the run's
own labels and the episodes that end in a goal restarted on the device, reported window by window (throughput, the
predictor's recall / precision on the window's decisions — its drift — and the result flags).

  python rocketsim-cuda_b200/rollout.py [--arenas 1048576] [--decisions 1000] [--retrain-every 64] [--mix contact]

Everything stays on the GPU between decisions: controls come from a pool of pre-uploaded sets (decision d uses set
d mod K), the predictor's training samples are drawn on the device from the features and labels of the decisions
themselves, and resets use rsx_reset_arenas_raw with the decision's result words (seed: reset_seed + d).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import rsx  # noqa: E402
import predictor as P  # noqa: E402


class Rollout:
    def __init__(self, runner, controls_pool, reset_seed: int, mix, config: dict, sample_per_decision: int = 32768, seed: int = 0):
        import torch

        self.t = torch
        self.run = runner
        self.pool = controls_pool
        self.reset_seed = reset_seed
        self.mix = (ctypes.c_float * 5)(*mix)
        self.config = dict(config)
        self.sample = min(sample_per_decision, runner.n)
        self.gen = torch.Generator(device=runner.dev.device)
        self.gen.manual_seed(seed)
        self.reset_count = torch.zeros(1, dtype=torch.int32, device=runner.dev.device)

    def run_decisions(self, decisions: int, retrain_every: int = 64, first: int = 0, on_decision=None, epochs: int = 2):
        """Decisions first .. first + decisions - 1; returns one record per window of retrain_every decisions."""
        t, run = self.t, self.run
        n = run.n
        dev = run.dev.device
        windows = []
        buf_x, buf_y = [], []
        tp = fp = fn = 0
        flags = {"scored": 0, "overflow": 0, "unimplemented": 0}
        ev0, ev1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        window_ms, window_dec, w_start = 0.0, 0, first
        with t.cuda.stream(run.stream):
            for d in range(first, first + decisions):
                cp = self.pool[d % len(self.pool)].data_ptr()
                ev0.record(run.stream)
                run.step(cp, self.config)
                self.reset_count.zero_()
                rsx.check(rsx.lib().rsx_reset_arenas_raw(run.ds.ptr(), n, run.dsd.ptr(), run.didx.data_ptr(), self.reset_seed + d, self.mix,
                                                         run.res.data_ptr(), None, self.reset_count.data_ptr(), run.sptr), "reset")
                ev1.record(run.stream)
                # labels of this decision, the predictor's guesses made before it, and training samples
                Y = run.pred.labels(run.ev.data_ptr(), n)
                if self.config["mode"] in ("binned", "levels"):
                    guess = (run.Z[:, :P.LABELS] > 0.0).any(dim=1)
                    truth = Y != 0
                    tp += int((guess & truth).sum())
                    fp += int((guess & ~truth).sum())
                    fn += int((~guess & truth).sum())
                pick = t.randint(0, n, (self.sample,), device=dev, generator=self.gen)
                buf_x.append(run.X.index_select(0, pick))
                buf_y.append(Y.index_select(0, pick))
                r = run.res.view(t.int32)
                flags["scored"] += int(((r & 0xFF) != 0).sum())
                flags["overflow"] += int(((r >> 30) & 1).sum())
                flags["unimplemented"] += int(((r >> 31) & 1).sum())
                ev1.synchronize()
                window_ms += ev0.elapsed_time(ev1)
                window_dec += 1
                if on_decision is not None:
                    on_decision(d)
                if window_dec == retrain_every or d == first + decisions - 1:
                    rec = {"decisions": [w_start, d], "ms_per_decision": window_ms / window_dec,
                           "arena_ticks_per_s": n * 8 * window_dec / (window_ms / 1e3),
                           "recall": tp / max(1, tp + fn), "precision": tp / max(1, tp + fp), **flags}
                    t0 = time.perf_counter()
                    X = t.cat(buf_x)
                    Yc = t.cat(buf_y)
                    run.pred.fit(X, Yc, epochs=epochs, batch=8192, lr=1e-3, seed=d)
                    run.stream.synchronize()
                    rec["retrain_s"] = time.perf_counter() - t0
                    windows.append(rec)
                    buf_x, buf_y = [], []
                    tp = fp = fn = 0
                    flags = {"scored": 0, "overflow": 0, "unimplemented": 0}
                    window_ms, window_dec, w_start = 0.0, 0, d + 1
        return windows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--arenas", type=int, default=1048576)
    ap.add_argument("--decisions", type=int, default=1000)
    ap.add_argument("--retrain-every", type=int, default=64)
    ap.add_argument("--mix", default="contact", choices=["contact", "headline"])
    ap.add_argument("--pool", type=int, default=16, help="control sets cycled through")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--order", default="levels", choices=["levels", "binned"],
                    help="the learned order: 16 cost levels (several claim rounds) or two bins")
    args = ap.parse_args()
    import torch

    sys.path.insert(0, os.path.dirname(HERE))
    import bench
    from runner import DecisionRunner

    mix = rsx.MIX_CONTACT_HEAVY if args.mix == "contact" else rsx.MIX_HEADLINE
    n = args.arenas
    dev = rsx.SimDevice(0)
    sds = np.stack([rsx.build_static(7, p, q) for p, q in bench.PRESETS])
    with np.errstate(over="ignore"):
        h = rsx._mix64(np.arange(n, dtype=np.uint64) + np.uint64(1 << 40))
    idx = (h % np.uint64(len(bench.PRESETS))).astype(np.uint8)
    st = rsx.make_states_multi(sds, idx, args.seed, mix)
    run = DecisionRunner(dev, sds, idx, st)
    del st
    pool = [torch.from_numpy(rsx.decision_controls(args.seed * 1000, k, n).view(np.int32)).to(dev.device) for k in range(args.pool)]
    t0 = time.perf_counter()
    run.train_predictor(control_seed=args.seed * 1000 + 500, decisions=max(2, 2097152 // n))
    train_s = time.perf_counter() - t0
    cfg = {"mode": args.order, "block": 448, "grid": run.sms, "split": 15, "threshold": 0.5}
    if args.order == "levels":
        cfg.update({"levels": 16, "weights": [1.0] * 6})
    ro = Rollout(run, pool, reset_seed=args.seed * 7919, mix=mix, config=cfg)
    windows = ro.run_decisions(args.decisions, args.retrain_every)
    total_ms = sum(w["ms_per_decision"] * (w["decisions"][1] - w["decisions"][0] + 1) for w in windows)
    print(json.dumps({"arenas": n, "decisions": args.decisions, "mix": args.mix, "order": args.order, "retrain_every": args.retrain_every,
                      "initial_train_s": round(train_s, 2), "arena_ticks_per_s": n * 8 * args.decisions / (total_ms / 1e3),
                      "windows": [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in w.items()} for w in windows]}))


if __name__ == "__main__":
    main()
