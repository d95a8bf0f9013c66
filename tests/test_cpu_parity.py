"""CPU-side parity of the simulator source against the oracle (the reference's own correctly rounded CPU build).

The simulator's single source compiles for the host too (rsx_host_phase / rsx_host_decide: -ffp-contract=off, no FMA
target, the same correctly rounded libm), so these tests check the arithmetic of every phase word for word without a
GPU; the GPU tests then check the device build against the same oracle.
"""
import ctypes

import numpy as np
import pytest


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def test_layout_sizes_match_reference(rsx, oracle):
    L = rsx.lib()
    assert L.rsx_arena_words() == oracle.L.lf_arena_words() == 2784
    assert L.rsx_tick_words() == oracle.L.lf_tick_words() == 2567
    assert L.rsx_static_words() == oracle.L.lf_static_words() == 317895
    for n in (1, 31, 32, 33, 1000):
        assert L.rsx_aosoa_words(n) == oracle.L.lf_aosoa_words(n)
    for a, w in [(0, 0), (1, 0), (31, 2783), (32, 0), (33, 5), (1000, 1234)]:
        assert L.rsx_aosoa_index(a, w) == oracle.L.lf_aosoa_index(a, w)


def test_pack_unpack_match_library(rsx, world):
    st = rsx.make_states(world, 45, 3)
    words = rsx.pack(st)
    ref = np.zeros(rsx.aosoa_words(45), np.uint32)
    rsx.lib().rsx_aosoa_pack(_p(st), 45, _p(ref))
    assert np.array_equal(words, ref)
    assert np.array_equal(rsx.unpack(words, 45), st)


@pytest.mark.parametrize("mix", ["headline", "contact"])
def test_every_phase_matches_oracle(rsx, oracle, world, mix):
    m = rsx.MIX_HEADLINE if mix == "headline" else rsx.MIX_CONTACT_HEAVY
    st = rsx.make_states(world, 24, 5, m)
    L = rsx.lib()
    for a in range(st.shape[0]):
        s = st[a].copy()
        for t in range(6):
            ctl = rsx.decision_controls(9, t, st.shape[0])[a]
            # controls are set before P0 (set_car_controls): write them into both cars' Controls words
            s[CTRL0:CTRL0 + 8] = ctl[:8]
            s[CTRL1:CTRL1 + 8] = ctl[8:]
            for k in range(10):
                want, got = s.copy(), s.copy()
                oracle.phase(k, want, world)
                L.rsx_host_phase(k, _p(got), _p(world))
                diff = np.nonzero(want != got)[0]
                assert diff.size == 0, f"arena {a} tick {t} phase {k}: words {diff[:8]}"
                s = want


@pytest.mark.parametrize("presets,mix,seed", [((0, 0), "kickoff", 1), ((0, 0), "headline", 2), ((4, 6), "contact", 3)])
def test_decisions_match_oracle(rsx, oracle, presets, mix, seed):
    sd = rsx.build_static(7, *presets)
    m = {"kickoff": rsx.MIX_KICKOFF, "headline": rsx.MIX_HEADLINE, "contact": rsx.MIX_CONTACT_HEAVY}[mix]
    st = rsx.make_states(sd, 48, seed, m)
    L = rsx.lib()
    for d in range(12):
        ctl = rsx.decision_controls(seed, d, 48)
        for a in range(48):
            want, got = st[a].copy(), st[a].copy()
            scored = oracle.decide(want, sd, ctl[a])
            res = L.rsx_host_decide(_p(got), _p(sd), _p(np.ascontiguousarray(ctl[a])))
            assert (res & 0xFF) == scored
            assert np.array_equal(want, got), f"arena {a} decision {d}"
            st[a] = want


# word offsets of cars[i].controls in ArenaState: tick_count 2 + rng 2 + ball 20 words, then the cars (247 words each);
# within a Car, controls follow dodge_deadzone 1, vel_impulse_cache 3, sticky_gate_prev 1, pos 3, rot 9, vel 3, ang_vel 3
CAR_WORDS = 247
CTRL0 = 24 + 23
CTRL1 = 24 + CAR_WORDS + 23
