"""Batched decisions on one GPU: the decision kernels, the learned binning in front of them, CUDA-graph capture of many
decisions, and the autotuner that picks the launch configuration.

A `DecisionRunner` owns the device buffers of one batch of arenas (AoSoA-32 states, per-arena car pairing, results,
event words, queue counter, arena order, predictor features and logits) and issues one decision with `step()`:

  sim8        k_sim8 through rsx_sim8_raw: the reference's sim8 entry (one StaticData for all arenas, block 32)
  plain       k_sim8_multi, one thread per arena, one launch per decision (the reference's sim8 shape, block 32)
  persistent  the persistent kernel without barriers (rsx_sim8_persistent_ex): register budget and queue granularity
  lockstep    the SM-lockstep persistent kernel (rsx_sim8_lockstep_ex) over the identity order, 8 / `ticks` launches
              of `ticks` ticks per decision (default 8: one launch)
  binned      the same kernel over the contact predictor's order: features -> MLP -> heavy/quiet bins -> order
  levels      the same kernel over the predictor's cost levels: features -> MLP -> 16 expected-contact levels -> order

Every configuration computes the same words (no cross-arena arithmetic), so the autotuner may pick any of them by
time alone; `tune()` restores the same start states before each candidate so that all candidates step identical work.
"""
from __future__ import annotations

import ctypes
import itertools

import numpy as np

import rsx
import predictor as P


class DecisionRunner:
    def __init__(self, dev: "rsx.SimDevice", statics: np.ndarray, sd_index: np.ndarray, states: np.ndarray, stream=None):
        import torch

        self.torch = torch
        self.dev = dev
        self.n = states.shape[0]
        self.stream = stream if stream is not None else torch.cuda.Stream(device=dev.device)
        self.sptr = self.stream.cuda_stream
        self.statics_host = np.ascontiguousarray(statics.reshape(-1, rsx.STATIC_WORDS), np.uint32)
        self.dsd = dev.upload_static(statics)
        self.ds = dev.upload_states(states)
        n = self.n
        t = torch
        self.didx = t.from_numpy(np.ascontiguousarray(sd_index, dtype=np.uint8)).to(dev.device)
        self.res = t.zeros(n, dtype=t.int32, device=dev.device)
        self.ev = t.zeros(n, dtype=t.int32, device=dev.device)
        self.counter = t.zeros(1, dtype=t.int32, device=dev.device)
        self.order = t.zeros(n, dtype=t.int32, device=dev.device)
        self.heavy = t.zeros(1, dtype=t.int32, device=dev.device)
        self.bin_scratch = t.zeros((n + 1023) // 1024, dtype=t.int32, device=dev.device)
        self.level_scratch = t.zeros(1 + 32 * ((n + 1023) // 1024), dtype=t.int32, device=dev.device)
        self.X = t.zeros((n, P.FEATURES), dtype=t.int16, device=dev.device)
        self.Z = t.zeros((n, 8), dtype=t.float32, device=dev.device)
        self.sms = torch.cuda.get_device_properties(dev.device).multi_processor_count
        self.pred = None
        self.config = {"mode": "lockstep", "block": 448, "grid": self.sms, "split": 15, "threshold": None}
        torch.cuda.synchronize(dev.device)

    # ---- observations and rewards of the last decision ----
    def observe(self, weights) -> tuple:
        """Launches rsx_observe_raw on the runner's stream over the current states, the last decision's result words
        and event OR: returns (obs (2n, 104) int16 holding FP16 bits, reward (2n,) float32), device tensors reused by
        later calls."""
        t = self.torch
        if not hasattr(self, "obs"):
            self.obs = t.zeros((2 * self.n, rsx.OBS_DIM), dtype=t.int16, device=self.dev.device)
            self.reward = t.zeros(2 * self.n, dtype=t.float32, device=self.dev.device)
            self.mirror = t.from_numpy(rsx.pad_mirror(self.statics_host).reshape(-1)).to(self.dev.device)
        w = (ctypes.c_float * rsx.REWARD_TERMS)(*[float(x) for x in weights])
        rsx.check(rsx.lib().rsx_observe_raw(self.ds.ptr(), self.n, self.dsd.ptr(), self.didx.data_ptr(), self.mirror.data_ptr(),
                                            self.res.data_ptr(), self.ev.data_ptr(), w, self.obs.data_ptr(), self.reward.data_ptr(),
                                            self.sptr), "rsx_observe_raw")
        return self.obs, self.reward

    # ---- one decision ----
    def step(self, controls_ptr: int, config: dict | None = None) -> None:
        c = config or self.config
        L = rsx.lib()
        n = self.n
        if c["mode"] == "sim8":  # the reference-shaped entry point: the first StaticData for every arena
            rsx.check(L.rsx_sim8_raw(self.ds.ptr(), n, self.dsd.ptr(), controls_ptr, self.res.data_ptr(), c.get("block", 32), None,
                                     self.sptr), "rsx_sim8_raw")
            return
        if c["mode"] == "plain":
            rsx.check(L.rsx_sim8_multi_raw(self.ds.ptr(), n, self.dsd.ptr(), self.didx.data_ptr(), controls_ptr, self.res.data_ptr(),
                                           self.ev.data_ptr(), c.get("block", 32), self.sptr), "rsx_sim8_multi_raw")
            return
        if c["mode"] == "persistent":  # the persistent kernel without barriers: register budget, queue granularity
            rsx.check(L.rsx_sim8_persistent_ex(self.ds.ptr(), n, self.dsd.ptr(), self.didx.data_ptr(), controls_ptr, self.res.data_ptr(),
                                               self.ev.data_ptr(), None, self.counter.data_ptr(), c["grid"], c["block"], c["granularity"],
                                               c["min_blocks"], None, self.sptr), "rsx_sim8_persistent_ex")
            return
        order = None
        if c["mode"] == "levels":
            p = self.pred
            w = (ctypes.c_float * P.LABELS)(*[float(x) for x in c.get("weights", [1.0] * P.LABELS)])
            rsx.check(p.L.rsx_pred_features_raw(self.ds.ptr(), n, self.dsd.ptr(), self.didx.data_ptr(), controls_ptr, self.X.data_ptr(),
                                                self.sptr), "features")
            p.logits(self.X, n, out=self.Z)
            rsx.check(p.L.rsx_pred_levels_raw(self.Z.data_ptr(), n, w, c.get("levels", 16), self.level_scratch.data_ptr(),
                                              self.order.data_ptr(), self.sptr), "levels")
            order = self.order.data_ptr()
        if c["mode"] == "binned":
            p = self.pred
            thr = float(np.log(c["threshold"] / (1.0 - c["threshold"])))
            rsx.check(p.L.rsx_pred_features_raw(self.ds.ptr(), n, self.dsd.ptr(), self.didx.data_ptr(), controls_ptr, self.X.data_ptr(),
                                                self.sptr), "features")
            p.logits(self.X, n, out=self.Z)
            rsx.check(p.L.rsx_pred_bin_raw(self.Z.data_ptr(), n, thr, c.get("labels", P.ALL_LABELS), self.bin_scratch.data_ptr(),
                                           self.order.data_ptr(), self.heavy.data_ptr(), self.sptr), "bin")
            order = self.order.data_ptr()
        rsx.check(L.rsx_sim8_lockstep_ex(self.ds.ptr(), n, self.dsd.ptr(), self.didx.data_ptr(), controls_ptr, self.res.data_ptr(),
                                         self.ev.data_ptr(), order, self.counter.data_ptr(), c.get("grid", self.sms), c["block"],
                                         c["split"], c.get("ticks", 8), self.sptr), "rsx_sim8_lockstep_ex")

    def kernels_per_step(self, config: dict | None = None) -> int:
        """This library's kernel launches per decision (features, forward, two binning passes or three level passes,
        and the decision's launches: 8 / ticks per launch for the lockstep kernel)."""
        c = config or self.config
        launches = 8 // c.get("ticks", 8) if c["mode"] in ("lockstep", "binned", "levels") else 1
        return {"binned": 4, "levels": 5}.get(c["mode"], 0) + launches

    # ---- states ----
    def snapshot(self):
        """A device copy of the states (restored by restore())."""
        t = self.torch
        words = rsx.aosoa_words(self.n)
        buf = t.empty(words, dtype=t.int32, device=self.dev.device)
        rsx.check(rsx.lib().rsx_copy_raw(buf.data_ptr(), self.ds.ptr(), words * 4, self.sptr), "rsx_copy_raw")
        self.stream.synchronize()  # the copy is complete for readers on any stream
        return buf

    def restore(self, buf) -> None:
        rsx.check(rsx.lib().rsx_copy_raw(self.ds.ptr(), buf.data_ptr(), rsx.aosoa_words(self.n) * 4, self.sptr), "rsx_copy_raw")

    # ---- the learned part ----
    def use_predictor(self, pred) -> None:
        """Takes a predictor trained elsewhere (another runner's, say), bound to this runner's stream so that its
        kernels stay ordered with this runner's features, binning passes and decisions."""
        self.pred = None if pred is None else pred.on_stream(self.sptr)

    def train_predictor(self, control_seed: int, decisions: int = 32, epochs: int = 6, seed: int = 0, lr: float = 2e-3):
        """Labels from `decisions` exact decisions of these arenas (controls of `control_seed`, run on a snapshot that is
        restored afterwards), then Adam over them; returns (samples, last losses)."""
        t = self.torch
        if self.pred is None:
            self.pred = P.ContactPredictor(self.dev.device, seed=seed, stream=self.sptr)
        snap = self.snapshot()
        Xs, Ys = [], []
        cfg = {"mode": "lockstep", "block": 448, "grid": self.sms, "split": 15}
        for d in range(decisions):
            ctl = t.from_numpy(rsx.decision_controls(control_seed, d, self.n).view(np.int32)).to(self.dev.device, non_blocking=False)
            self.stream.wait_stream(t.cuda.current_stream(self.dev.device))
            X = t.empty((self.n, P.FEATURES), dtype=t.int16, device=self.dev.device)
            Y = t.empty(self.n, dtype=t.uint8, device=self.dev.device)
            rsx.check(self.pred.L.rsx_pred_features_raw(self.ds.ptr(), self.n, self.dsd.ptr(), self.didx.data_ptr(), ctl.data_ptr(),
                                                        X.data_ptr(), self.sptr), "features")
            self.step(ctl.data_ptr(), cfg)
            rsx.check(self.pred.L.rsx_pred_labels_raw(self.ev.data_ptr(), self.n, Y.data_ptr(), self.sptr), "labels")
            self.stream.synchronize()
            Xs.append(X)
            Ys.append(Y)
        self.restore(snap)
        self.stream.synchronize()
        X, Y = t.cat(Xs), t.cat(Ys)
        with t.cuda.stream(self.stream):
            losses = []
            for ep in range(epochs):
                losses = self.pred.fit(X, Y, epochs=1, batch=8192, lr=lr, seed=seed + ep)
        self.stream.synchronize()
        return X.shape[0], losses

    # ---- the autotuner ----
    def candidates(self, binning: bool = True):
        # the plain launch too: with few arenas per SM (a few thousand arenas) the barriers cost more than they save
        out = [{"mode": "plain", "block": 32}, {"mode": "plain", "block": 64}]
        # the persistent kernel without barriers: register budget (min_blocks of 64 threads per SM) and queue granularity
        for min_blocks, gran in ((8, 1), (8, 4), (12, 1)):
            out.append({"mode": "persistent", "block": 64, "grid": self.sms * min_blocks, "granularity": gran, "min_blocks": min_blocks})
        # splits: 7 (lockstep), 14 (+ P3b's mesh-leaf tests, the SATs' feature pairs and the wheel rays' mesh leaves
        # pooled over the block, P3a in one piece), 15 (14 with the wheel rays' mesh walks pooled too)
        for block, split in itertools.product((448, 512), (7, 14, 15)):
            out.append({"mode": "lockstep", "block": block, "grid": self.sms, "split": split, "threshold": None})
            if split == 15:  # ticks per launch: a decision in 2 or 4 launches, arenas re-claimed (re-balanced) between them
                for ticks in (4, 2):
                    out.append({"mode": "lockstep", "block": block, "grid": self.sms, "split": split, "threshold": None, "ticks": ticks})
            if binning and self.pred is not None and split >= 14:
                for thr, labels in ((0.3, P.ALL_LABELS), (0.5, P.ALL_LABELS)):
                    out.append({"mode": "binned", "block": block, "grid": self.sms, "split": split, "threshold": thr, "labels": labels})
                out.append({"mode": "levels", "block": block, "grid": self.sms, "split": split, "threshold": None, "levels": 16,
                            "weights": [1.0] * P.LABELS})
        return out

    def tune(self, controls_ptrs, candidates=None, repeats: int = 1, margin: float = 0.01):
        """Times every candidate on the same decisions from the same start states, `repeats` times each (the candidates
        interleaved round by round, so that a slow stretch of the machine does not fall on one candidate) and ranks
        them by median time (one lucky repeat does not decide; with one repeat the median is that time).  Keeps as
        self.config, among the candidates within `margin` of the best median, the one with the fewest kernel launches
        per decision (a difference inside the run-to-run spread does not buy the predictor's extra launches).  Returns
        [(median ms, config, [ms of every repeat])] sorted by median time."""
        t = self.torch
        snap = self.snapshot()
        cands = list(candidates or self.candidates())
        times = [[] for _ in cands]
        for _ in range(repeats):
            for i, c in enumerate(cands):
                self.restore(snap)
                e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
                e0.record(self.stream)
                for cp in controls_ptrs:
                    self.step(cp, c)
                e1.record(self.stream)
                e1.synchronize()
                times[i].append(e0.elapsed_time(e1))
        self.restore(snap)
        self.stream.synchronize()
        results = sorted(((sorted(ts)[(len(ts) - 1) // 2], c, ts) for ts, c in zip(times, cands)), key=lambda r: r[0])
        close = [r for r in results if r[0] <= results[0][0] * (1.0 + margin)]
        self.config = dict(min(close, key=lambda r: (self.kernels_per_step(r[1]), r[0]))[1])
        return results

    # ---- CUDA graphs ----
    def capture(self, controls_ptrs, config: dict | None = None):
        """One CUDA graph of len(controls_ptrs) consecutive decisions (each with its own controls buffer)."""
        t = self.torch
        g = t.cuda.CUDAGraph()
        self.stream.synchronize()
        with t.cuda.graph(g, stream=self.stream):
            for cp in controls_ptrs:
                self.step(cp, config)
        return g

    def replay(self, g) -> None:
        """Replays a captured graph on this runner's stream (torch replays on the current stream)."""
        with self.torch.cuda.stream(self.stream):
            g.replay()

    def free(self):
        self.ds.free()
        self.dsd.free()
