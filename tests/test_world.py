"""Invariants of the synthetic world (StaticData) and of the seeded start states (a consistent broadphase)."""
import numpy as np
import pytest

STATIC_COUNTS = dict(tris=8020, nodes=3754, leaves=8020, cells=242, cell_entries=1210)


def test_static_builds_for_every_preset(rsx):
    for p0 in range(7):
        for p1 in range(7):
            if p0 != p1 and (p0 + p1) % 3:
                continue
            sd = rsx.build_static(7, p0, p1)
            assert sd.shape == (rsx.STATIC_WORDS,)


def test_static_is_deterministic_and_seeded(rsx):
    a, b, c = rsx.build_static(7, 0, 0), rsx.build_static(7, 0, 0), rsx.build_static(8, 0, 0)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)


def test_states_are_deterministic(rsx, world):
    a, b = rsx.make_states(world, 64, 5), rsx.make_states(world, 64, 5)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, rsx.make_states(world, 64, 6))
    assert np.all(a[:, rsx.TICK_WORDS:] == 0), "the mid-tick part of a start state is zero"


# broadphase words: handle_edges at 2311 (24 x 3 words of u16 lo[3], hi[3]), edges at 2383 (3 x 48 words of u16 pos,
# handle), n_pairs at 2527, pairs at 2528 (16 x 2)
HE, ED, NP, PR = 2311, 2383, 2527, 2528


@pytest.mark.parametrize("mix", ["headline", "contact"])
def test_start_broadphase_is_consistent(rsx, world, mix):
    m = rsx.MIX_HEADLINE if mix == "headline" else rsx.MIX_CONTACT_HEAVY
    st = rsx.make_states(world, 128, 9, m)
    for s in st:
        he = s[HE:HE + 72].view(np.uint16).reshape(24, 6)
        ed = s[ED:ED + 144].view(np.uint16).reshape(3, 48, 2)
        for ax in range(3):
            pos = ed[ax, :, 0].astype(np.int64)
            assert np.all(np.diff(pos) >= 0), "edges sorted along each axis"
            assert ed[ax, 0, 1] == 0 and ed[ax, 47, 1] == 0, "sentinels at both ends"
            for h in range(1, 24):
                lo, hi = he[h, ax], he[h, 3 + ax]
                assert ed[ax, lo, 1] == h and ed[ax, hi, 1] == h and lo < hi
                assert ed[ax, lo, 0] % 2 == 0 and ed[ax, hi, 0] % 2 == 1
        n = int(s[NP])
        pairs = {tuple(s[PR + 2 * i:PR + 2 * i + 2]) for i in range(n)}
        assert len(pairs) == n
        for a, b in pairs:
            assert a < b
            for ax in range(3):
                assert he[a, 3 + ax] > he[b, ax] and he[b, 3 + ax] > he[a, ax], "a retained pair overlaps on every axis"


def test_one_decision_keeps_start_states_in_caps(rsx, world):
    st = rsx.make_states(world, 64, 4, rsx.MIX_CONTACT_HEAVY)
    import ctypes

    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))  # noqa: E731
    for d in range(4):
        ctl = rsx.decision_controls(4, d, 64)
        for a in range(64):
            r = rsx.lib().rsx_host_decide(p(st[a]), p(world), p(np.ascontiguousarray(ctl[a])))
            assert (r & (rsx.OVERFLOW | rsx.UNIMPLEMENTED)) == 0
