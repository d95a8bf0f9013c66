"""The contact predictor (host side): a small MLP that guesses, from an arena's state at decision start, which kinds of
contact its next 8 ticks will have, and turns the guesses into an arena order for the persistent decision kernels
(contact-heavy arenas first, then quiet ones).

Everything numeric runs in the library's kernels (include/rsx.h, rsx_pred_*): features, forward, backward, Adam and
binning.  torch tensors are only device buffers here.  The network: 48 features -> 128 -> 128 -> 128 (ReLU) -> 6
sigmoid outputs, BF16 weights and activations with FP32 accumulation, FP32 master weights for Adam.  Labels are the
decision's event OR (bit 0 car 0 - ball, 1 car 1 - ball, 2 car - car, 3 ball - world, 4 car 0 - world, 5 car 1 - world).

Scheduling only: the decision kernels' results do not depend on the order, so predictions cost time, never
correctness; recall and precision are measured against the exact labels the simulator produces.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

import rsx

FEATURES = 48
LABELS = 6
HIDDEN = 128
PARAMS = 40328
# outputs: 0 car 0 - ball, 1 car 1 - ball, 2 car - car, 3 ball - world, 4 car 0 - world, 5 car 1 - world
ALL_LABELS = 0x3F
CAR_LABELS = 0x37  # every output but ball - world
# offsets of the parameter blocks (floats)
OFF = {}
_o = 0
for _name, _size in [("W1", HIDDEN * FEATURES), ("b1", HIDDEN), ("W2", HIDDEN * HIDDEN), ("b2", HIDDEN), ("W3", HIDDEN * HIDDEN),
                     ("b3", HIDDEN), ("W4", 8 * HIDDEN), ("b4", 8)]:
    OFF[_name] = (_o, _size)
    _o += _size
assert _o == PARAMS


def _bind():
    L = rsx.lib()
    if getattr(L, "_pred_bound", False):
        return L
    vp, u32 = ctypes.c_void_p, ctypes.c_uint32
    L.rsx_pred_features_raw.argtypes = [vp, u32, vp, vp, vp, vp, vp]
    L.rsx_pred_labels_raw.argtypes = [vp, u32, vp, vp]
    L.rsx_pred_forward_raw.argtypes = [vp, vp, vp, u32, vp, vp]
    L.rsx_pred_scratch_elems.argtypes = [u32]
    L.rsx_pred_scratch_elems.restype = ctypes.c_uint64
    L.rsx_pred_gradients_raw.argtypes = [vp, vp, vp, vp, u32, vp, vp, vp, vp, vp]
    L.rsx_pred_adam_raw.argtypes = [vp, vp, vp, vp, vp, u32, ctypes.c_float, vp]
    L.rsx_pred_to_bf16_raw.argtypes = [vp, vp, vp]
    L.rsx_pred_bin_raw.argtypes = [vp, u32, ctypes.c_float, u32, vp, vp, vp, vp]
    L.rsx_pred_levels_raw.argtypes = [vp, u32, ctypes.POINTER(ctypes.c_float), u32, vp, vp, vp]
    L.rsx_pred_forward_tc_raw.argtypes = [vp, vp, vp, u32, vp, vp, vp]
    L._pred_bound = True
    return L


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights (fan-in), zero biases; rows 6 and 7 of W4 zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)
    for name, shape, live in [("W1", (HIDDEN, FEATURES), HIDDEN), ("W2", (HIDDEN, HIDDEN), HIDDEN), ("W3", (HIDDEN, HIDDEN), HIDDEN),
                              ("W4", (8, HIDDEN), LABELS)]:
        o, size = OFF[name]
        lim = math.sqrt(6.0 / shape[1])
        w = np.zeros(shape, np.float32)
        w[:live] = rng.uniform(-lim, lim, size=(live, shape[1])).astype(np.float32)
        p[o:o + size] = w.reshape(-1)
    return p


def unpack_params(p: np.ndarray) -> dict:
    """The parameter blocks as arrays: W1 (128, 48), b1, W2 (128, 128), b2, W3, b3, W4 (8, 128), b4 (8)."""
    shapes = {"W1": (HIDDEN, FEATURES), "W2": (HIDDEN, HIDDEN), "W3": (HIDDEN, HIDDEN), "W4": (8, HIDDEN)}
    return {k: p[o:o + s].reshape(shapes.get(k, (s,))) for k, (o, s) in OFF.items()}


class ContactPredictor:
    """Weights and optimiser state on one device; every call is asynchronous on `stream` (a cudaStream_t or None)."""

    def __init__(self, device, seed: int = 0, stream=None):
        import torch

        self.torch = torch
        self.device = device
        self.stream = stream
        self.L = _bind()
        self.w = torch.from_numpy(init_params(seed)).to(device)
        self.wb = torch.zeros(PARAMS, dtype=torch.int16, device=device)
        self.m = torch.zeros(PARAMS, dtype=torch.float32, device=device)
        self.v = torch.zeros(PARAMS, dtype=torch.float32, device=device)
        self.grad = torch.zeros(PARAMS, dtype=torch.float32, device=device)
        self.loss = torch.zeros(1, dtype=torch.float32, device=device)
        self.step = 0
        self._scratch = None
        self._scratch_n = 0
        torch.cuda.synchronize(device)
        rsx.check(self.L.rsx_pred_to_bf16_raw(self.w.data_ptr(), self.wb.data_ptr(), self.stream), "rsx_pred_to_bf16_raw")

    # ---- data ----
    def features(self, d_states: int, n: int, d_statics: int, d_sd_index: int, d_controls: int, out=None):
        t = self.torch
        X = out if out is not None else t.empty((n, FEATURES), dtype=t.int16, device=self.device)
        rsx.check(self.L.rsx_pred_features_raw(d_states, n, d_statics, d_sd_index, d_controls, X.data_ptr(), self.stream),
                  "rsx_pred_features_raw")
        return X

    def labels(self, d_event_or: int, n: int, out=None):
        t = self.torch
        Y = out if out is not None else t.empty(n, dtype=t.uint8, device=self.device)
        rsx.check(self.L.rsx_pred_labels_raw(d_event_or, n, Y.data_ptr(), self.stream), "rsx_pred_labels_raw")
        return Y

    def on_stream(self, stream) -> "ContactPredictor":
        """The same network (weights and optimiser state shared, not copied) issuing its kernels on `stream`.  A caller
        whose other kernels run on another stream must use such a view: the binning and level orders are counting sorts
        in two or three passes over the logits, and logits written on one stream while a pass on another reads them can
        place an arena past the end of the order.  Train through one view only (the Adam step count is the view's)."""
        import copy

        self.torch.cuda.synchronize(self.device)  # what this view's stream issued so far is done before the other starts
        v = copy.copy(self)
        v.stream = stream
        v._scratch, v._scratch_n = None, 0
        return v

    # ---- network ----
    def logits(self, X, n: int, out=None):
        """Inference on the tensor cores (tcgen05: rsx_pred_forward_tc_raw)."""
        t = self.torch
        Z = out if out is not None else t.empty((n, 8), dtype=t.float32, device=self.device)
        if not hasattr(self, "tc_error"):
            self.tc_error = t.zeros(1, dtype=t.int32, device=self.device)
        rsx.check(self.L.rsx_pred_forward_tc_raw(self.wb.data_ptr(), self.w.data_ptr(), X.data_ptr(), n, Z.data_ptr(),
                                                 self.tc_error.data_ptr(), self.stream), "rsx_pred_forward_tc_raw")
        return Z

    def logits_mma_sync(self, X, n: int, out=None):
        """The same forward on mma.sync (the training kernels' forward)."""
        t = self.torch
        Z = out if out is not None else t.empty((n, 8), dtype=t.float32, device=self.device)
        rsx.check(self.L.rsx_pred_forward_raw(self.wb.data_ptr(), self.w.data_ptr(), X.data_ptr(), n, Z.data_ptr(), self.stream),
                  "rsx_pred_forward_raw")
        return Z

    def _scratch_for(self, n: int):
        if self._scratch is None or self._scratch_n < n:
            t = self.torch
            self._scratch = t.empty(int(self.L.rsx_pred_scratch_elems(n)), dtype=t.int16, device=self.device)
            self._logits = t.empty((n, 8), dtype=t.float32, device=self.device)
            self._scratch_n = n
        return self._scratch

    def gradients(self, X, Y, n: int):
        """Gradients of the mean (over the batch) summed binary cross-entropy into self.grad; self.loss = n * loss."""
        scratch = self._scratch_for(n)
        rsx.check(self.L.rsx_pred_gradients_raw(self.wb.data_ptr(), self.w.data_ptr(), X.data_ptr(), Y.data_ptr(), n, scratch.data_ptr(),
                                                self._logits.data_ptr(), self.grad.data_ptr(), self.loss.data_ptr(), self.stream),
                  "rsx_pred_gradients_raw")
        return self.grad

    def train_step(self, X, Y, n: int, lr: float = 1e-3):
        self.gradients(X, Y, n)
        self.step += 1
        rsx.check(self.L.rsx_pred_adam_raw(self.w.data_ptr(), self.wb.data_ptr(), self.m.data_ptr(), self.v.data_ptr(), self.grad.data_ptr(),
                                           self.step, lr, self.stream), "rsx_pred_adam_raw")

    def fit(self, X, Y, epochs: int = 2, batch: int = 8192, lr: float = 1e-3, seed: int = 0):
        """Adam over shuffled minibatches of (X [N][48] BF16 words, Y [N] label bytes); returns the last batch losses."""
        t = self.torch
        N = X.shape[0]
        g = t.Generator(device="cpu")
        g.manual_seed(seed)
        losses = []
        for _ in range(epochs):
            perm = t.randperm(N, generator=g).to(self.device)
            for b0 in range(0, N - batch + 1, batch):
                idx = perm[b0:b0 + batch]
                xb = X.index_select(0, idx).contiguous()
                yb = Y.index_select(0, idx).contiguous()
                self.train_step(xb, yb, batch, lr)
                losses.append(self.loss)
                self.loss = t.zeros(1, dtype=t.float32, device=self.device)
        return [float(l.item()) / batch for l in losses[-8:]]

    # ---- binning ----
    def bin(self, Z, n: int, threshold: float = 0.5, order=None, heavy=None, label_mask: int = 0x3F):
        """Order of the arenas for the persistent kernels: predicted contact-heavy first (any output of label_mask above
        the threshold), then quiet (each in arena order)."""
        t = self.torch
        order = order if order is not None else t.empty(n, dtype=t.int32, device=self.device)
        heavy = heavy if heavy is not None else t.zeros(1, dtype=t.int32, device=self.device)
        scratch = t.empty((n + 1023) // 1024, dtype=t.int32, device=self.device)
        thr = math.log(threshold / (1.0 - threshold))
        rsx.check(self.L.rsx_pred_bin_raw(Z.data_ptr(), n, thr, label_mask, scratch.data_ptr(), order.data_ptr(), heavy.data_ptr(), self.stream),
                  "rsx_pred_bin_raw")
        return order, heavy

    def params(self) -> np.ndarray:
        return self.w.cpu().numpy()


def recall_precision(Z: np.ndarray, Y: np.ndarray, threshold: float = 0.5):
    """Per label and for "any contact": (recall, precision, positive rate) of logits Z [n][8] against label bytes Y [n]."""
    thr = math.log(threshold / (1.0 - threshold))
    pred = Z[:, :LABELS] > thr
    truth = ((Y[:, None] >> np.arange(LABELS)) & 1).astype(bool)
    out = {}
    for k, name in enumerate(["car0_ball", "car1_ball", "car_car", "ball_world", "car0_world", "car1_world"]):
        tp = np.sum(pred[:, k] & truth[:, k])
        out[name] = (tp / max(1, truth[:, k].sum()), tp / max(1, pred[:, k].sum()), float(truth[:, k].mean()))
    pa, ta = pred.any(1), truth.any(1)
    tp = np.sum(pa & ta)
    out["any"] = (tp / max(1, ta.sum()), tp / max(1, pa.sum()), float(ta.mean()))
    return out
