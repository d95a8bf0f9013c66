"""Test infrastructure: a NumPy restatement of the observation and reward kernel (rsx_observe_raw, k_observe), the
oracle its GPU test compares against bit for bit.  Only tests import this file.

The reference defines no observation (its RL training loop is not part of it); it ships the FP16 conversion such a
kernel uses (cuda/common/hd.cuh:167-176: round to nearest even), which NumPy's float32 -> float16 cast also is.  The
layout and the reward terms are the ones include/rsx.h fixes.  Field offsets come from the reference's own structure
layout as restated in oracle/v3dump.py (by field name), not from this project's headers.  Every FP32 operation is a
NumPy float32 elementwise operation (round to nearest, never fused) in the kernel's order.
"""
from __future__ import annotations

import numpy as np

import v3dump as L

OBS_DIM = 104
REWARD_TERMS = 8
POS = np.float32(1) / np.float32(2300)
ANG = np.float32(1 / np.pi)
BOOST = np.float32(0.01)
TICK = np.float32(1) / np.float32(120)
EV_CAR_HIT_BALL, EV_BUMP, EV_DEMO, EV_PICKUP = 0, 2, 4, 6

A = L.ARENA_STATE.fields
C = L.CAR.fields


def _w(off_bytes):
    return off_bytes // 4


def _car(c, name, sub=None):
    off = A["cars"][0] + c * L.CAR.size + C[name][0]
    if sub is not None:
        off += L.MAT3.fields[sub][0]
    return _w(off)


def _f(S, w, k=3):
    return S[:, w:w + k].view(np.float32)


def _half(x):
    return np.asarray(x, np.float32).astype(np.float16).view(np.uint16)


def pad_mirror(sd_words: np.ndarray) -> np.ndarray:
    v = sd_words.view(np.float32)
    base = _w(L.STATIC_DATA.fields["pads"][0])
    size = _w(L.PAD_CONST.size)
    pos = np.stack([v[base + p * size:base + p * size + 3] for p in range(L.NUM_PADS)])
    out = np.arange(L.NUM_PADS, dtype=np.uint8)
    for p in range(L.NUM_PADS):
        m = np.array([-pos[p, 0], -pos[p, 1], pos[p, 2]], np.float32)
        hit = np.nonzero(np.all(pos == m, axis=1))[0]
        if hit.size:
            out[p] = hit[0]
    return out


def observe(states, sds, sd_index, mirror, result, event_or, weights):
    """states (n, 2784) u32; sds (count, 317895); sd_index (n,); mirror (count, 34) or None; result / event_or (n,) or
    None; weights (8,) f32.  Returns obs (2n, 104) u16 bits and reward (2n,) f32."""
    S = np.ascontiguousarray(states, np.uint32)
    n = S.shape[0]
    si = np.asarray(sd_index, np.int64) if sd_index is not None else np.zeros(n, np.int64)
    res = np.zeros(n, np.uint32) if result is None else np.asarray(result, np.uint32)
    ev = np.zeros(n, np.uint32) if event_or is None else np.asarray(event_or, np.uint32)
    wt = np.asarray(weights, np.float32)
    sdf = sds.view(np.float32)
    pad_base, pad_size = _w(L.STATIC_DATA.fields["pads"][0]), _w(L.PAD_CONST.size)
    cool_off = _w(L.PAD_CONST.fields["max_cooldown"][0])
    cooldown = np.stack([sdf[si, pad_base + p * pad_size + cool_off] for p in range(L.NUM_PADS)], axis=1)
    team_of = np.stack([sds[si, _w(L.STATIC_DATA.fields["cars"][0] + c * L.CAR_CONST.size + L.CAR_CONST.fields["team"][0])]
                        for c in range(2)], axis=1)

    bpos = _f(S, _w(A["ball"][0] + L.BALL_DYN.fields["pos"][0]))
    bvel = _f(S, _w(A["ball"][0] + L.BALL_DYN.fields["vel"][0]))
    bang = _f(S, _w(A["ball"][0] + L.BALL_DYN.fields["ang_vel"][0]))
    tick = (S[:, _w(A["tick_count"][0]) + 1].astype(np.uint64) << np.uint64(32) | S[:, _w(A["tick_count"][0])]).astype(np.int64)
    active = np.ones((n, L.NUM_PADS), bool)
    for p in range(L.NUM_PADS):
        w = _w(A["pad_gave_boost"][0]) + p * 3
        some = S[:, w] != 0
        last = (S[:, w + 2].astype(np.uint64) << np.uint64(32) | S[:, w + 1]).astype(np.int64)
        elapsed = (tick - last).astype(np.float32) * TICK
        active[:, p] = ~some | ~(elapsed < cooldown[:, p])

    obs = np.zeros((n, 2, OBS_DIM), np.uint16)
    reward = np.zeros((n, 2), np.float32)
    for c in range(2):
        o = 1 - c
        sgn = np.array([-1, -1, 1] if c else [1, 1, 1], np.float32)  # negation is exact

        def put(k, v, scale):
            obs[:, c, k:k + 3] = _half((v * sgn) * scale)

        def put_diff(k, a, b, scale):
            obs[:, c, k:k + 3] = _half(((a - b) * sgn) * scale)

        pos, vel, ang = _f(S, _car(c, "pos")), _f(S, _car(c, "vel")), _f(S, _car(c, "ang_vel"))
        fwd, up = _f(S, _car(c, "rot_mat", "x_axis")), _f(S, _car(c, "rot_mat", "z_axis"))
        opos, ovel, oang = _f(S, _car(o, "pos")), _f(S, _car(o, "vel")), _f(S, _car(o, "ang_vel"))
        ofwd, oup = _f(S, _car(o, "rot_mat", "x_axis")), _f(S, _car(o, "rot_mat", "z_axis"))
        put(0, bpos, POS)
        put(3, bvel, POS)
        put(6, bang, ANG)
        put(9, pos, POS)
        put(12, fwd, np.float32(1))
        put(15, up, np.float32(1))
        put(18, vel, POS)
        put(21, ang, ANG)
        obs[:, c, 24] = _half(_f(S, _car(c, "boost"), 1)[:, 0] * BOOST)
        for k, name in enumerate(("is_on_ground", "has_jumped", "has_double_jumped", "has_flipped", "is_demoed")):
            obs[:, c, 25 + k] = _half(S[:, _car(c, name)] != 0)
        put_diff(30, bpos, pos, POS)
        put_diff(33, bvel, vel, POS)
        put(36, opos, POS)
        put(39, ofwd, np.float32(1))
        put(42, oup, np.float32(1))
        put(45, ovel, POS)
        put(48, oang, ANG)
        obs[:, c, 51] = _half(_f(S, _car(o, "boost"), 1)[:, 0] * BOOST)
        obs[:, c, 52] = _half(S[:, _car(o, "is_on_ground")] != 0)
        obs[:, c, 53] = _half(S[:, _car(o, "is_demoed")] != 0)
        put_diff(54, opos, pos, POS)
        put_diff(57, ovel, vel, POS)
        ctl = _car(c, "controls")
        obs[:, c, 60:65] = _half(_f(S, ctl, 5))
        obs[:, c, 65:68] = _half(S[:, ctl + 5:ctl + 8] != 0)
        if c and mirror is not None:
            q = np.asarray(mirror, np.int64)[si]
            obs[:, c, 68:102] = _half(np.take_along_axis(active, q, axis=1))
        else:
            obs[:, c, 68:102] = _half(active)

        team = team_of[:, c]
        scored = (res & 0xFF) != 0
        goal = np.where(scored, np.where((bpos[:, 1] > 0) == (team == 0), np.float32(1), np.float32(-1)), np.float32(0))
        d = bpos - pos
        length = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
        dot = (vel[:, 0] * d[:, 0] + vel[:, 1] * d[:, 1]) + vel[:, 2] * d[:, 2]
        with np.errstate(divide="ignore", invalid="ignore"):
            toward = np.where(length > 0, (dot / length) * POS, np.float32(0))
        ball_goal = np.where(team == 0, bvel[:, 1], -bvel[:, 1]) * POS

        def bit(k):
            return ((ev >> np.uint32(k)) & np.uint32(1)).astype(np.float32)
        terms = [goal, bit(EV_CAR_HIT_BALL + c), bit(EV_BUMP + o), bit(EV_DEMO + o), bit(EV_DEMO + c), bit(EV_PICKUP + c),
                 toward, ball_goal]
        total = wt[0] * terms[0].astype(np.float32)
        for k in range(1, REWARD_TERMS):
            total = total + wt[k] * terms[k].astype(np.float32)
        reward[:, c] = total
    return obs.reshape(2 * n, OBS_DIM), reward.reshape(2 * n)
