"""GPU parity: the sm_100a kernels against the oracle (the reference's own correctly rounded CPU build), word for word
on every tick-boundary state word and every result, through the C ABI.  Where the oracle library is absent the
committed golden fixtures (tests/golden/decisions.json, libm_chunk_hashes.json, made from the oracle) stand in."""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, ORACLE_SO, Oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev(rsx):
    d = rsx.SimDevice(0)
    yield d
    d.close()


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def oracle_or_none():
    return Oracle() if os.path.exists(ORACLE_SO) else None


def test_upload_download_and_identity_kernels(rsx, dev, world):
    import torch

    st = rsx.make_states(world, 77, 3)
    st[:, rsx.TICK_WORDS:] = np.arange(rsx.ARENA_WORDS - rsx.TICK_WORDS, dtype=np.uint32)  # mid-tick words too
    ds = dev.upload_states(st)
    assert np.array_equal(dev.download_states(ds), st)
    out = torch.zeros(rsx.aosoa_words(77), dtype=torch.int32, device=dev.device)
    for tick_only in (0, 1):
        out.zero_()
        rsx.check(rsx.lib().rsx_identity(dev.h, ds.ptr(), out.data_ptr(), 77, tick_only), "identity")
        dev.sync()
        back = rsx.unpack(out.cpu().numpy().view(np.uint32), 77)
        want = st.copy()
        if tick_only:
            want[:, rsx.TICK_WORDS:] = 0
        assert np.array_equal(back, want)
    ds.free()


def run_case_gpu(rsx, dev, case, oracle):
    sd = rsx.build_static(case["world_seed"], *case["presets"])
    assert sha(sd) == case["static_sha"], "the synthetic world generator changed"
    st = rsx.make_states(sd, case["n"], case["state_seed"], tuple(case["mix"]))
    assert sha(st) == case["init_sha"], "the start-state generator changed"
    n = case["n"]
    dsd = dev.upload_static(sd)
    ds = dev.upload_states(st)
    res = dev.alloc_result(n)
    ref = st.copy() if oracle else None
    for d in range(case["decisions"]):
        ctl = rsx.decision_controls(case["control_seed"], d, n)
        dev.sim8(ds, dsd, dev.upload_controls(ctl), res)
        got = dev.download_states(ds)
        r = res.cpu().numpy().view(np.uint32)
        assert not np.any(r & (rsx.OVERFLOW | rsx.UNIMPLEMENTED))
        if oracle:
            scored = oracle.run(ref, sd, ctl)
            bad = np.nonzero(np.any(got[:, :rsx.TICK_WORDS] != ref[:, :rsx.TICK_WORDS], axis=1))[0]
            assert bad.size == 0, f"decision {d}: arenas {bad[:8]} differ from the oracle"
            assert np.array_equal(r & 0xFF, scored)
        assert sha((r & 0xFF).astype(np.uint32), got[:, :rsx.TICK_WORDS]) == case["per_decision"][d], f"decision {d}"
    ds.free()
    dsd.free()


def golden_cases():
    with open(os.path.join(GOLDEN, "decisions.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("idx", range(4))
def test_sim8_matches_oracle(rsx, dev, idx):
    case = golden_cases()[idx]
    run_case_gpu(rsx, dev, case, oracle_or_none())


def test_result_independent_of_block_order_and_queue(rsx, dev):
    """Block 32 vs 64, the multi-static kernel, the persistent kernel over a permuted order with several queue
    granularities, and the SM-lockstep kernel over several grids, blocks, barrier splits and orders (grid 2 x 64
    threads: 4 warps take 32 claims in turn) give the same words (the reference's determinism test,
    tests/step.rs:455-506)."""
    import torch

    sds = np.stack([rsx.build_static(7, p, q) for p, q in [(0, 0), (1, 2), (5, 6)]])
    n = 1000
    idx = (np.arange(n) % 3).astype(np.uint8)
    st = np.zeros((n, rsx.ARENA_WORDS), np.uint32)
    rsx.check(rsx.lib().rsx_make_states_multi(rsx._p(sds.reshape(-1)), 3, idx.ctypes.data_as(ctypes.c_void_p), rsx._p(st), n, 5,
                                               (ctypes.c_float * 5)(*rsx.MIX_CONTACT_HEAVY)), "make_states_multi")
    dsd = dev.upload_static(sds)
    didx = torch.from_numpy(idx).to(dev.device)
    outs = []
    perm = np.random.default_rng(1).permutation(n).astype(np.uint32)
    dperm = torch.from_numpy(perm.view(np.int32)).to(dev.device)
    counter = torch.zeros(1, dtype=torch.int32, device=dev.device)
    variants = [("multi", 32, None, 0, 0), ("multi", 64, None, 0, 0), ("persist", 32, dperm, 148, 1), ("persist", 64, dperm, 37, 3),
                ("persist", 32, None, 7, 2), ("lock", 512, dperm, 148, 1), ("lock", 384, None, 3, 0), ("lock", 448, dperm, 2, 1),
                ("lock", 64, dperm, 2, 1), ("lock", 480, None, 1, 0), ("lock", 448, dperm, 148, 2),
                ("lock", 96, None, 2, 2), ("lock", 512, dperm, 148, 3), ("lock", 64, None, 3, 3),
                ("lock", 448, dperm, 148, 6), ("lock", 96, None, 2, 6), ("lock", 448, None, 148, 4), ("lock", 64, dperm, 2, 5),
                ("lock", 448, dperm, 148, 7), ("lock", 448, dperm, 148, 9), ("lock", 96, None, 2, 9), ("lock", 512, None, 5, 9),
                ("lock", 448, dperm, 148, 10), ("lock", 64, None, 3, 10), ("lock", 448, dperm, 148, 11), ("lock", 96, None, 2, 11),
                ("lock", 512, None, 5, 11), ("lock", 448, dperm, 148, 14), ("lock", 64, None, 3, 14), ("lock", 512, None, 5, 14),
                ("lock", 448, dperm, 148, 15), ("lock", 96, None, 2, 15), ("lock", 512, None, 5, 15)]
    for kind, block, order, grid, gran in variants:
        ds = dev.upload_states(st)
        res = dev.alloc_result(n)
        ev = torch.zeros(n, dtype=torch.int32, device=dev.device)
        for d in range(6):
            ctl = dev.upload_controls(rsx.decision_controls(3, d, n))
            if kind == "multi":
                rc = rsx.lib().rsx_sim8_multi_raw(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), res.data_ptr(), ev.data_ptr(),
                                                  block, dev.stream_ptr())
            elif kind == "lock":
                rc = rsx.lib().rsx_sim8_lockstep_raw(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), res.data_ptr(), ev.data_ptr(),
                                                     order.data_ptr() if order is not None else None, counter.data_ptr(), grid, block, gran,
                                                     dev.stream_ptr())
            else:
                rc = rsx.lib().rsx_sim8_persistent_raw(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), res.data_ptr(), ev.data_ptr(),
                                                       order.data_ptr() if order is not None else None, counter.data_ptr(), grid, block,
                                                       gran, dev.stream_ptr())
            rsx.check(rc, kind)
        dev.sync()
        outs.append((dev.download_states(ds), res.cpu().numpy(), ev.cpu().numpy()))
        ds.free()
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0])
        assert np.array_equal(o[1], outs[0][1])
        assert np.array_equal(o[2], outs[0][2])
    # and against the oracle, arena by arena with its own car pairing
    orc = oracle_or_none()
    if orc:
        ref = st.copy()
        for d in range(6):
            ctl = rsx.decision_controls(3, d, n)
            for a in range(n):
                orc.decide(ref[a], sds[idx[a]], ctl[a])
        assert np.array_equal(ref[:, :rsx.TICK_WORDS], outs[0][0][:, :rsx.TICK_WORDS])


def test_ticks_per_launch_same_words(rsx, dev):
    """A decision split over 2, 4 or 8 launches of the lockstep kernel (rsx_sim8_lockstep_ex; progress carried in the
    result and event words, arenas re-claimed between launches) gives the words of the one-launch decision: states,
    result words (goals included: a scored arena keeps its goal state through the later launches) and event words, over
    several claim rounds (grid 2) and one (grid 148), identity and permuted orders."""
    import torch

    sds = np.stack([rsx.build_static(7, p, q) for p, q in [(0, 0), (2, 6)]])
    n = 1000
    idx = (np.arange(n) % 2).astype(np.uint8)
    st = rsx.make_states_multi(sds, idx, 17, rsx.MIX_CONTACT_HEAVY)
    dsd = dev.upload_static(sds)
    didx = torch.from_numpy(idx).to(dev.device)
    perm = torch.from_numpy(np.random.default_rng(4).permutation(n).astype(np.int32)).to(dev.device)
    counter = torch.zeros(1, dtype=torch.int32, device=dev.device)
    L = rsx.lib()
    outs = []
    for ticks, grid, order, block in ((8, 148, None, 448), (4, 148, None, 448), (2, 2, perm, 448), (1, 148, perm, 512), (4, 3, None, 64)):
        ds = dev.upload_states(st)
        res = dev.alloc_result(n)
        ev = torch.zeros(n, dtype=torch.int32, device=dev.device)
        scored = 0
        for d in range(6):
            ctl = dev.upload_controls(rsx.decision_controls(13, d, n))
            rsx.check(L.rsx_sim8_lockstep_ex(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), res.data_ptr(), ev.data_ptr(),
                                             order.data_ptr() if order is not None else None, counter.data_ptr(), grid, block, 15, ticks,
                                             dev.stream_ptr()), f"lockstep ticks {ticks}")
            dev.sync()
            scored += int(((res.cpu().numpy().view(np.uint32) & 0xFF) != 0).sum())
        outs.append((dev.download_states(ds)[:, :rsx.TICK_WORDS], res.cpu().numpy(), ev.cpu().numpy(), scored))
        ds.free()
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0])
        assert np.array_equal(o[1], outs[0][1])
        assert np.array_equal(o[2], outs[0][2])
    assert outs[0][3] > 0, "the case should hold goals (a scored arena must keep its goal state across launches)"
    assert L.rsx_sim8_lockstep_ex(None, n, dsd.ptr(), None, None, None, None, None, None, 148, 448, 7, 3, None) == -1
    dsd.free()


def test_trace_and_tick_kernels_match_oracle(rsx, dev, world):
    import torch

    orc = oracle_or_none()
    if orc is None:
        pytest.skip("needs the oracle library")
    n = 96
    st = rsx.make_states(world, n, 8, rsx.MIX_CONTACT_HEAVY)
    ctl = rsx.decision_controls(8, 0, n)
    ds = dev.upload_states(st)
    dsd = dev.upload_static(world)
    trace = torch.zeros(8 * rsx.aosoa_words(n), dtype=torch.int32, device=dev.device)
    res = dev.alloc_result(n)
    dev.sim8(ds, dsd, dev.upload_controls(ctl), res, trace=trace)
    dev.sync()
    tr = trace.cpu().numpy().view(np.uint32).reshape(8, -1)
    r = res.cpu().numpy().view(np.uint32)
    for a in range(n):
        s = st[a].copy()
        want = np.zeros((8, rsx.ARENA_WORDS), np.uint32)
        sc = ctypes.c_uint32(0)
        orc.L.rscuda_step_ticks(orc.p(s), orc.p(world), orc.p(np.ascontiguousarray(ctl[a])), 8, ctypes.byref(sc), orc.p(want))
        upto = sc.value if sc.value else 8
        for t in range(upto):
            got = rsx.unpack(tr[t], n)[a]
            assert np.array_equal(got[:rsx.TICK_WORDS], want[t][:rsx.TICK_WORDS]), f"arena {a} tick {t + 1}"
        assert (r[a] & 0xFF) == sc.value
    # one tick and single phases through their kernels
    from test_cpu_parity import CTRL0, CTRL1

    st2 = st.copy()
    st2[:, CTRL0:CTRL0 + 8] = ctl[:, :8]
    st2[:, CTRL1:CTRL1 + 8] = ctl[:, 8:]
    ds2 = dev.upload_states(st2)
    status = dev.step_tick(ds2, dsd)
    assert np.all(status == 0)
    got = dev.download_states(ds2)
    for a in range(n):
        s = st2[a].copy()
        orc.L.rscuda_step_tick(orc.p(s), orc.p(world))
        assert np.array_equal(got[a][:rsx.TICK_WORDS], s[:rsx.TICK_WORDS])
    cur = st2.copy()
    ds3 = dev.upload_states(cur)
    for k in range(10):
        dev.phase(k, ds3, dsd)
        got = dev.download_states(ds3)
        for a in range(n):
            orc.phase(k, cur[a], world)
        assert np.array_equal(got, cur), f"phase {k}"


@pytest.mark.parametrize("fn,name", [(0, "sin"), (1, "cos"), (2, "tan")])
def test_libm_all_inputs_on_device(rsx, dev, fn, name):
    """All 2^32 binary32 inputs of the device's correctly rounded sin / cos / tan, hashed by 2^24-input chunks, equal
    the reference's correctly rounded values (hashes made on a CPU from the reference's libm)."""
    import torch

    with open(os.path.join(GOLDEN, "libm_chunk_hashes.json")) as f:
        gold = json.load(f)[name]
    L = rsx.lib()
    L.rsx_libm_chunk_hashes.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    h = torch.zeros(256, dtype=torch.int64, device=dev.device)
    rsx.check(L.rsx_libm_chunk_hashes(fn, 0, 256, h.data_ptr(), dev.stream_ptr()), "libm hashes")
    dev.sync()
    got = ["%016x" % (int(v) & 0xFFFFFFFFFFFFFFFF) for v in h.cpu().numpy()]
    bad = [c for c in range(256) if got[c] != gold[c]]
    assert not bad, f"{name}: chunks {bad[:10]} differ"
