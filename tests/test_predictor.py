"""The contact predictor: its kernels against a NumPy FP32 restatement of the same network (BF16 rounding of weights
and activations emulated at the points the kernels round), its gradients against finite differences of that
restatement, the feature and label kernels against NumPy from the unpacked states, and the binning kernel's order.

Tolerances (BF16 has an 8-bit significand, 2^-8 relative rounding error): features within one BF16 step; logits and
every gradient block within 2% relative (L2 norm of the difference over the norm of the reference), since FP32 sums in
a different order can move an intermediate BF16 value by one step."""
import ctypes
import math

import numpy as np
import pytest

import predictor as P


def bf16(x):
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = (b + np.uint32(0x7FFF) + ((b >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000)
    return r.view(np.float32)


def from_bf16_words(w):
    return (np.asarray(w).astype(np.uint16).astype(np.uint32) << np.uint32(16)).view(np.float32)


def reference(p, X, Y, round_bf16=True):
    """Forward and backward of the predictor in NumPy FP32: (logits [n][8], grads dict, loss)."""
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, np.float32))
    w = P.unpack_params(p)
    W = {k: r(w[k]) for k in ("W1", "W2", "W3", "W4")}
    n = X.shape[0]
    x = r(X)
    h1 = r(np.maximum(x @ W["W1"].T + w["b1"], 0))
    h2 = r(np.maximum(h1 @ W["W2"].T + w["b2"], 0))
    h3 = r(np.maximum(h2 @ W["W3"].T + w["b3"], 0))
    z = (h3 @ W["W4"].T + w["b4"]).astype(np.float32)
    y = ((Y[:, None] >> np.arange(8)) & 1).astype(np.float32)
    y[:, 6:] = 0
    p_ = 1.0 / (1.0 + np.exp(-z))
    dz = (p_ - y) / np.float32(n)
    dz[:, 6:] = 0
    dz = r(dz)
    loss = np.sum((np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))[:, :6]) / n
    g3 = r((dz @ W["W4"]) * (h3 > 0))
    g2 = r((g3 @ W["W3"]) * (h2 > 0))
    g1 = r((g2 @ W["W2"]) * (h1 > 0))
    grads = {"W4": dz.T @ h3, "b4": dz.sum(0), "W3": g3.T @ h2, "b3": g3.sum(0), "W2": g2.T @ h1, "b2": g2.sum(0), "W1": g1.T @ x,
             "b1": g1.sum(0)}
    return z, grads, np.float32(loss)


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / max(1e-12, np.linalg.norm(b.ravel())))


def test_reference_gradients_match_finite_differences():
    """The restatement's backward pass (FP32, no BF16 rounding) against central differences of its loss."""
    rng = np.random.default_rng(3)
    p = P.init_params(5) * np.float32(0.5)
    p[P.OFF["b1"][0]:P.OFF["b1"][0] + 128] = rng.normal(0, 0.1, 128).astype(np.float32)
    X = rng.normal(0, 1, (24, 48)).astype(np.float32)
    Y = rng.integers(0, 64, 24).astype(np.uint8)
    _, g, _ = reference(p, X, Y, round_bf16=False)
    eps = np.float32(2e-3)
    for name, picks in [("W1", [(3, 7), (100, 40)]), ("W2", [(5, 9), (77, 120)]), ("W3", [(0, 0), (64, 31)]), ("W4", [(2, 17), (5, 99)]),
                        ("b1", [(11,)]), ("b4", [(4,)])]:
        o, size = P.OFF[name]
        shape = g[name].shape
        for ij in picks:
            flat = o + (np.ravel_multi_index(ij, shape) if len(shape) > 1 else ij[0])
            q = p.copy()
            q[flat] += eps
            lp = reference(q, X, Y, round_bf16=False)[2]
            q[flat] -= 2 * eps
            lm = reference(q, X, Y, round_bf16=False)[2]
            fd = (lp - lm) / (2 * eps)
            an = g[name][ij]
            assert abs(fd - an) <= 2e-3 + 5e-2 * abs(an), f"{name}{ij}: finite difference {fd} vs analytic {an}"


def test_recall_precision_counts():
    Z = np.full((4, 8), -5.0, np.float32)
    Z[0, 0] = 5.0  # predicted car0-ball
    Z[1, 3] = 5.0  # predicted ball-world
    Y = np.array([1, 0, 8, 0], np.uint8)  # true car0-ball on 0, ball-world on 2
    m = P.recall_precision(Z, Y)
    assert m["car0_ball"][:2] == (1.0, 1.0)
    assert m["ball_world"][:2] == (0.0, 0.0)
    assert m["any"][:2] == (0.5, 0.5)


# ---- GPU ----
def _world(rsx, n, seed=4):
    sds = np.stack([rsx.build_static(7, p, q) for p, q in [(0, 0), (2, 5), (6, 3)]])
    idx = (np.arange(n) % 3).astype(np.uint8)
    st = rsx.make_states_multi(sds, idx, seed, rsx.MIX_HEADLINE)
    return sds, idx, st


def _features_np(st, ctl):
    """The 48 features from unpacked states (word offsets of the reference's ArenaState: ball at word 4, cars at word
    24 + 247 i; within a Car pos +5, rot +8 (column c2 at +14), vel +17, ang_vel +20, boost +44, on_ground +62)."""
    f = st.view(np.float32)
    n = st.shape[0]
    out = np.zeros((n, 48), np.float32)
    bp, bv, bw = f[:, 4:7], f[:, 16:19], f[:, 19:22]
    out[:, 0:3] = bp * np.float32(1 / 4096)
    out[:, 3:6] = bv * np.float32(1 / 6000)
    out[:, 6:9] = bw * np.float32(1 / 6)
    cp, cv = [], []
    for c in range(2):
        b = 24 + 247 * c
        g = 9 + 14 * c
        cp.append(f[:, b + 5:b + 8])
        cv.append(f[:, b + 17:b + 20])
        out[:, g:g + 3] = cp[c] * np.float32(1 / 4096)
        out[:, g + 3:g + 6] = cv[c] * np.float32(1 / 2300)
        out[:, g + 6:g + 9] = f[:, b + 20:b + 23] * np.float32(1 / 5.5)
        out[:, g + 9:g + 12] = f[:, b + 14:b + 17]
        out[:, g + 12] = (st[:, b + 62] != 0).astype(np.float32)
        out[:, g + 13] = f[:, b + 44] * np.float32(0.01)
    d = lambda p, q: np.sqrt(np.sum((p - q) ** 2, axis=1))
    dcc = d(cp[0], cp[1])
    out[:, 37] = dcc / 4096
    out[:, 38] = d(cp[0], bp) / 4096
    out[:, 39] = d(cp[1], bp) / 4096
    bd = lambda p: np.minimum(np.minimum(4096 - np.abs(p[:, 0]), 5120 - np.abs(p[:, 1])), np.minimum(p[:, 2], 2044 - p[:, 2]))
    out[:, 40] = bd(bp) * np.float32(0.001)
    out[:, 41] = bd(cp[0]) * np.float32(0.001)
    out[:, 42] = bd(cp[1]) * np.float32(0.001)
    out[:, 45] = (ctl[:, 5] != 0).astype(np.float32)
    out[:, 46] = (ctl[:, 13] != 0).astype(np.float32)
    rv = np.sum((cv[1] - cv[0]) * (cp[0] - cp[1]), axis=1)
    out[:, 47] = rv / np.maximum(dcc, 1) / 2300
    return out


@pytest.mark.gpu
def test_feature_and_label_kernels(rsx):
    import torch

    n = 300
    sds, idx, st = _world(rsx, n)
    dev = rsx.SimDevice(0)
    try:
        pr = P.ContactPredictor(dev.device)
        dsd = dev.upload_static(sds)
        ds = dev.upload_states(st)
        didx = torch.from_numpy(idx).to(dev.device)
        ctl = rsx.decision_controls(7, 0, n)
        dctl = dev.upload_controls(ctl)
        X = pr.features(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), dctl.data_ptr())
        torch.cuda.synchronize()
        got = from_bf16_words(X.cpu().numpy())
        want = bf16(_features_np(st, ctl))
        cols = [c for c in range(48) if c not in (43, 44)]
        step = np.float32(2.0 ** -7) * np.maximum(np.abs(want[:, cols]), np.float32(1e-30))
        bad = np.abs(got[:, cols] - want[:, cols]) > step + 1e-6
        assert not bad.any(), f"feature columns {sorted(set(np.array(cols)[np.nonzero(bad)[1]]))} differ"
        assert np.all(got[:, 43:45] >= 0) and np.all(got[:, 43:45] <= 4.1)
        # labels from a real decision's event OR
        res = dev.alloc_result(n)
        ev = torch.zeros(n, dtype=torch.int32, device=dev.device)
        rsx.check(rsx.lib().rsx_sim8_multi_raw(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), dctl.data_ptr(), res.data_ptr(), ev.data_ptr(), 32,
                                               dev.stream_ptr()), "multi")
        dev.sync()
        Y = pr.labels(ev.data_ptr(), n)
        torch.cuda.synchronize()
        e = ev.cpu().numpy().view(np.uint32)
        want_y = ((e & 1) | (e & 2) | np.where((e >> 2) & 15, 4, 0) | np.where(e & ((1 << 12) | (1 << 14)), 8, 0) | (((e >> 10) & 1) << 4) |
                  (((e >> 11) & 1) << 5)).astype(np.uint8)
        assert np.array_equal(Y.cpu().numpy(), want_y)
        ds.free()
        dsd.free()
    finally:
        dev.close()


@pytest.mark.gpu
def test_forward_and_gradients_match_reference():
    import torch

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(11)
    n = 1000  # not a multiple of 16: a partial last tile
    X = bf16(rng.normal(0, 1, (n, 48)).astype(np.float32))
    Y = rng.integers(0, 64, n).astype(np.uint8)
    pr = P.ContactPredictor(dev, seed=2)
    p = pr.params()
    Xw = torch.from_numpy((X.view(np.uint32) >> 16).astype(np.uint16).view(np.int16)).to(dev)
    Yd = torch.from_numpy(Y).to(dev)
    Z = pr.logits(Xw, n)
    pr.gradients(Xw, Yd, n)
    torch.cuda.synchronize()
    z_ref, g_ref, loss_ref = reference(p, X, Y)
    z = Z.cpu().numpy()
    assert rel(z[:, :6], z_ref[:, :6]) < 2e-2
    g = P.unpack_params(pr.grad.cpu().numpy())
    for k in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        assert rel(g[k], g_ref[k]) < 2e-2, f"gradient {k}: relative difference {rel(g[k], g_ref[k]):.4f}"
    assert abs(float(pr.loss.item()) / n - loss_ref) < 2e-2 * abs(loss_ref)


@pytest.mark.gpu
def test_training_lowers_loss_and_binning_orders_heavy_first():
    import torch

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(5)
    n = 8192
    Xf = rng.normal(0, 1, (n, 48)).astype(np.float32)
    # a learnable rule: label k set when feature k > 0.3
    Y = sum(((Xf[:, k] > 0.3).astype(np.uint8) << k) for k in range(6)).astype(np.uint8)
    X = torch.from_numpy((bf16(Xf).view(np.uint32) >> 16).astype(np.uint16).view(np.int16)).to(dev)
    Yd = torch.from_numpy(Y).to(dev)
    pr = P.ContactPredictor(dev, seed=1)
    losses = []
    for it in range(60):
        pr.train_step(X, Yd, n, lr=3e-3)
        losses.append(float(pr.loss.item()) / n)
    assert losses[-1] < 0.5 * losses[0], losses[::10]
    Z = pr.logits(X, n)
    order, heavy = pr.bin(Z, n, 0.5)
    torch.cuda.synchronize()
    z = Z.cpu().numpy()
    o = order.cpu().numpy()
    h = int(heavy.item())
    is_heavy = (z[:, :6] > 0).any(1)
    assert sorted(o.tolist()) == list(range(n))
    assert h == int(is_heavy.sum())
    assert np.all(is_heavy[o[:h]]) and not np.any(is_heavy[o[h:]])
    assert np.all(np.diff(o[:h]) > 0) and np.all(np.diff(o[h:]) > 0)
    m = P.recall_precision(z, Y)
    assert m["any"][0] > 0.9 and m["any"][1] > 0.9


@pytest.mark.gpu
def test_cost_levels_order_is_a_stable_descending_sort():
    """rsx_pred_levels_raw on logits of +-30 (each output's probability 0 or 1 to FP32 precision, so an arena's expected
    contact count is its number of set outputs k and, with 7 levels and the maximum 6, its level floor(7k / 6) lies far
    from a level boundary): the order is the stable sort by level, highest first, over several blocks."""
    import torch

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(9)
    n = 5000
    on = rng.random((n, 6)) < 0.3
    on[17] = True  # one arena with all six: the batch maximum is 6
    z = np.zeros((n, 8), np.float32)
    z[:, :6] = np.where(on, 30.0, -30.0)
    Z = torch.from_numpy(z).to(dev)
    order = torch.zeros(n, dtype=torch.int32, device=dev)
    scratch = torch.zeros(1 + 7 * ((n + 1023) // 1024), dtype=torch.int32, device=dev)
    import rsx

    L = P._bind()
    w = (ctypes.c_float * 6)(*([1.0] * 6))
    rsx.check(L.rsx_pred_levels_raw(Z.data_ptr(), n, w, 7, scratch.data_ptr(), order.data_ptr(), None), "levels")
    torch.cuda.synchronize()
    k = on.sum(1)
    level = np.minimum(k * 7 // 6, 6)
    want = np.argsort(-level, kind="stable")
    assert np.array_equal(order.cpu().numpy(), want)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 4099, 65536])
def test_tensor_core_forward_matches_mma_sync_forward(n):
    """rsx_pred_forward_tc_raw (tcgen05.mma, accumulators in tensor memory) against rsx_pred_forward_raw (mma.sync)
    on the same BF16 features and weights: the same BF16 products, FP32 sums in another order, and activations rounded
    to BF16 between layers in both, so the logits agree to within a few BF16 steps."""
    import torch

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(n)
    pr = P.ContactPredictor(dev, seed=7)
    Xf = rng.normal(0, 1, (n, 48)).astype(np.float32)
    X = torch.from_numpy((bf16(Xf).view(np.uint32) >> 16).astype(np.uint16).view(np.int16)).to(dev)
    ref = pr.logits_mma_sync(X, n).clone()
    got = torch.full_like(ref, float("nan"))
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    L = P._bind()
    rsx_mod = __import__("rsx")
    rsx_mod.check(L.rsx_pred_forward_tc_raw(pr.wb.data_ptr(), pr.w.data_ptr(), X.data_ptr(), n, got.data_ptr(), err.data_ptr(), None),
                  "forward_tc")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    r, g = ref.cpu().numpy()[:, :6], got.cpu().numpy()[:, :6]
    assert np.all(np.isfinite(g))
    scale = float(np.abs(r).max()) + 1e-6
    assert float(np.abs(g - r).max()) < 0.03 * scale, (float(np.abs(g - r).max()), scale)
    assert float(np.linalg.norm(g - r) / np.linalg.norm(r)) < 5e-3
