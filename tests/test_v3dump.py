"""V3 dump import / export (rsx_v3_*: the reference's crates/rocketsim-cuda/src/dump.rs) against the independent CPU
restatement of the format in oracle/v3dump.py: the same bytes out, the same words in, the same refusals with the
same messages.  Inputs are states of the synthetic world at tick boundaries (start states and after decisions) and in
the middle of ticks (after the narrowphase, with contact records, and after the island phase), stepped by the
library's host build of the simulator."""
import ctypes
import json
import os
import struct
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import v3dump as O  # noqa: E402

A = O.ARENA_STATE.fields
W_EVENTS = A["events"][0] // 4
W_OVERFLOW = A["overflow"][0] // 4
CTRL = [(A["cars"][0] + k * O.CAR.size + O.CAR.fields["controls"][0]) // 4 for k in range(2)]
NOT_IN_DUMP = [W_EVENTS] + list(range(W_OVERFLOW, W_OVERFLOW + 6))  # the tick's events and the overflow counters


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def _in_dump(words):
    w = words.copy()
    w[NOT_IN_DUMP] = 0
    return w


@pytest.fixture(scope="module")
def cases(rsx):
    """(state words, static words, label): tick-boundary and mid-tick states of three car pairings and two mixes."""
    L = rsx.lib()
    out = []
    for presets, mix, seed in [((0, 0), rsx.MIX_HEADLINE, 3), ((4, 6), rsx.MIX_CONTACT_HEAVY, 5), ((2, 3), rsx.MIX_CONTACT_HEAVY, 9)]:
        sd = rsx.build_static(7, *presets)
        st = rsx.make_states(sd, 10, seed, mix)
        for a in range(st.shape[0]):
            out.append((st[a].copy(), sd, f"start {presets} {a}"))
        for d in range(4):
            ctl = rsx.decision_controls(seed, d, st.shape[0])
            for a in range(st.shape[0]):
                L.rsx_host_decide(_p(st[a]), _p(sd), _p(np.ascontiguousarray(ctl[a])))
                out.append((st[a].copy(), sd, f"decision {d + 1} {presets} {a}"))
        ctl = rsx.decision_controls(seed, 99, st.shape[0])
        for a in range(st.shape[0]):
            s = st[a].copy()
            s[CTRL[0]:CTRL[0] + 8] = ctl[a][:8]
            s[CTRL[1]:CTRL[1] + 8] = ctl[a][8:]
            for k in range(6):  # P0 .. P4: after P3b (k = 4) the records are live, after P4 the active list
                L.rsx_host_phase(k, _p(s), _p(sd))
                if k >= 4:
                    out.append((s.copy(), sd, f"mid-tick after phase {k} {presets} {a}"))
    return out


def golden_states(rsx):
    """(label, state words, static words) of the pinned dumps: two start states, one after two decisions, one after the
    narrowphase of the next tick (contact records live), of one car pairing."""
    L = rsx.lib()
    sd = rsx.build_static(7, 4, 6)
    st = rsx.make_states(sd, 6, 11, rsx.MIX_CONTACT_HEAVY)
    out = [("start 0", st[0].copy(), sd), ("start 1", st[1].copy(), sd)]
    for d in range(2):
        ctl = rsx.decision_controls(11, d, 6)
        for a in range(6):
            L.rsx_host_decide(_p(st[a]), _p(sd), _p(np.ascontiguousarray(ctl[a])))
    out.append(("after 2 decisions, arena 2", st[2].copy(), sd))
    s = st[3].copy()
    for k in range(5):
        L.rsx_host_phase(k, _p(s), _p(sd))
    out.append(("after the narrowphase, arena 3", s, sd))
    return out


def test_dumps_match_the_pinned_hashes(rsx):
    """The committed sha256 of dumps of fixed states (tests/golden/make_v3_golden.py): both implementations reproduce them."""
    import hashlib

    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "v3dump.json")) as f:
        pinned = json.load(f)
    for (label, s, sd), want in zip(golden_states(rsx), pinned["arena"]):
        t = rsx.V3Template()
        t.config_hash, t.ball_other_set = 0x1234, 1
        got = rsx.v3_write_arena(s, sd, t)
        assert want["case"] == label and hashlib.sha256(got).hexdigest() == want["sha256"], label
        to = O.empty_template()
        to.update({"config_hash": 0x1234, "ball_other_set": True})
        assert hashlib.sha256(O.write_arena(s, sd, to)).hexdigest() == want["sha256"], label
    sb = rsx.v3_write_static(_full_static(rsx))
    assert hashlib.sha256(sb).hexdigest() == pinned["static"]["sha256"]
    assert f"{rsx.v3_config_hash(_full_static(rsx)):016x}" == pinned["static"]["config_hash"]


def test_fnv1a64_published_vectors(rsx):
    for data, h in [(b"", 0xCBF29CE484222325), (b"a", 0xAF63DC4C8601EC8C), (b"foobar", 0x85944171F73967E8)]:
        assert rsx.v3_fnv1a64(data) == h == O.fnv1a64(data)


def test_layout_and_record_sizes(rsx):
    assert O.ARENA_WORDS == rsx.ARENA_WORDS and O.TICK_WORDS == rsx.TICK_WORDS and O.STATIC_WORDS == rsx.STATIC_WORDS
    w = O.Wr()
    O.io_body(w, O.V(bytearray(O.BODY.size), 0, O.BODY))
    assert len(w.out) == 219  # BODY_RECORD_LEN (dump.rs:21)
    assert ctypes.sizeof(rsx.V3Template) == 5088


def test_cases_cover_every_list(cases):
    got = {"manifolds": 0, "pairs": 0, "dyn_cells": 0, "records": 0, "active": 0, "folded": 0, "pad_touch": 0}
    for s, _, _ in cases:
        v = O.V(bytearray(s.tobytes()), 0, O.ARENA_STATE)
        got["manifolds"] += v.n_manifolds > 0
        got["pairs"] += v.n_pairs > 0
        got["dyn_cells"] += v.n_dyn_cells > 0
        got["records"] += v.n_records > 0
        got["active"] += v.n_active > 0
        got["folded"] += v.fold_events != 0
        got["pad_touch"] += any(v.pad_touching[p].n for p in range(O.NUM_PADS))
    assert all(c > 0 for c in got.values()), got


def test_arena_export_matches_oracle_and_imports_back(rsx, cases):
    for s, sd, label in cases:
        t = rsx.v3_template(sd)
        b = rsx.v3_write_arena(s, sd, t)
        tpy = {"config_hash": t.config_hash, "static_body": [bytes(t.static_body[i]) for i in range(23)],
               "num_handles": t.num_handles, "next_new_handle": t.next_new_handle, "manifold_stride": t.manifold_stride,
               "ball_other": bytes(t.ball_other), "ball_other_set": bool(t.ball_other_set)}
        assert b == O.write_arena(s, sd, tpy), label
        got, t2 = rsx.v3_parse_arena(b, sd)
        ref, tref = O.parse_arena(b, sd)
        assert np.array_equal(got, ref), f"{label}: words {np.nonzero(got != ref)[0][:8]}"
        assert np.array_equal(got, _in_dump(s)), f"{label}: words {np.nonzero(got != _in_dump(s))[0][:8]}"
        assert [bytes(t2.static_body[i]) for i in range(23)] == tref["static_body"] == tpy["static_body"]
        assert (t2.num_handles, t2.next_new_handle, t2.config_hash) == (t.num_handles, t.next_new_handle, t.config_hash)
        assert rsx.v3_write_arena(got, sd, t2) == b, label  # a dump re-exported from its import is the same dump


def test_arena_header(rsx, cases):
    s, sd, _ = next(c for c in cases if O.V(bytearray(c[0].tobytes()), 0, O.ARENA_STATE).n_manifolds > 0)
    t = rsx.v3_template(sd)
    b = rsx.v3_write_arena(s, sd, t)
    assert b[:8] == b"V3ARENA\0" and struct.unpack_from("<I", b, 8)[0] == 2
    assert struct.unpack_from("<Q", b, 12)[0] == t.config_hash == rsx.v3_config_hash(sd)
    counts = struct.unpack_from("<12I", b, 20)
    v = O.V(bytearray(s.tobytes()), 0, O.ARENA_STATE)
    assert counts[0] == 23 and counts[1] == v.n_manifolds and counts[4] == 32 * 32 and counts[5] == 24
    assert counts[6] == v.n_pairs and counts[7] == v.n_dyn_cells and counts[8:10] == (2, 34)
    assert b[68:72] == b"ARNA"


def _first_offset(b, tag):
    return b.index(tag)


def _both_refuse(rsx, b, sd, msg):
    with pytest.raises(rsx.RsxError) as e:
        rsx.v3_parse_arena(b, sd)
    assert f"({O_E_FORMAT})" in str(e.value) and msg in str(e.value), str(e.value)
    with pytest.raises(O.DumpError) as e2:
        O.parse_arena(b, sd)
    assert str(e2.value) == msg


O_E_FORMAT = -5


def test_arena_refusals_match_oracle(rsx, cases):
    s, sd, _ = next(c for c in cases if O.V(bytearray(c[0].tobytes()), 0, O.ARENA_STATE).n_manifolds > 0)
    t = rsx.v3_template(sd)
    b = rsx.v3_write_arena(s, sd, t)
    _both_refuse(rsx, b"V3ARENX\0" + b[8:], sd, "not an arena dump (magic)")
    _both_refuse(rsx, b[:8] + struct.pack("<I", 1) + b[12:], sd, "unsupported arena dump version 1")
    _both_refuse(rsx, b + b"\0\0\0", sd, "3 trailing bytes")
    for cut in (69, 100, 2000, len(b) - 1):
        msgs = []
        with pytest.raises(rsx.RsxError) as e:
            rsx.v3_parse_arena(b[:cut], sd)
        with pytest.raises(O.DumpError) as e2:
            O.parse_arena(b[:cut], sd)
        assert str(e2.value) in str(e.value) and str(e2.value) in ("dump truncated", "count exceeds the bytes left"), (cut, str(e.value))
    ball_only = 68 + 4 + 16  # ARNA tag, tick count, rng
    _both_refuse(rsx, b[:ball_only] + b"\x01" + b[ball_only + 1:], sd, "a ball-only arena")
    ground_stick = b.index(b"CARS") - 1
    _both_refuse(rsx, b[:ground_stick] + b"\x01" + b[ground_stick + 1:], sd, "Snowday ground_stick_applied is set")
    disp = b.index(b"DISP") + 4
    _both_refuse(rsx, b[:disp] + struct.pack("<I", 17) + b[disp + 4:], sd, "retained manifolds over the cap")
    # the first manifold point's applied_impulse: 2 indices + key + 2 thresholds + count, then 5 vec3 + 3 floats
    applied = disp + 4 + 8 + 8 + 8 + 4 + 60 + 12
    _both_refuse(rsx, b[:applied] + struct.pack("<f", 1.0) + b[applied + 4:], sd, "manifold point with a non-zero applied_impulse")
    key = disp + 4 + 8
    _both_refuse(rsx, b[:key] + struct.pack("<Q", 5) + b[key + 8:], sd, "manifold pair_key is not min << 32 | max")
    # constants that differ from StaticData
    sd2 = sd.copy()
    v = O.V(bytearray(sd2.tobytes()), 0, O.STATIC_DATA)
    v.proxies[1].aabb.get("min").x = O.f32_bits(-12345.0)
    _both_refuse(rsx, b, np.frombuffer(bytes(v.b), np.uint32).copy(), "a static broadphase proxy differs from StaticData.proxies")
    v = O.V(bytearray(sd.tobytes()), 0, O.STATIC_DATA)
    v.proxies[2].unique_id = 999
    _both_refuse(rsx, b, np.frombuffer(bytes(v.b), np.uint32).copy(), "a broadphase proxy constant differs from StaticData.proxies")
    v = O.V(bytearray(sd.tobytes()), 0, O.STATIC_DATA)
    for i in range(23):
        v.bodies[i].contact_breaking_threshold = O.f32_bits(0.125)
    _both_refuse(rsx, b, np.frombuffer(bytes(v.b), np.uint32).copy(), "a manifold threshold is not the min over its two bodies")


def test_record_fold_overflow_refused(rsx, cases):
    """More car - ball / car - car records than the cap: both refuse, as the reference's fold does (overflow[2])."""
    s, sd, _ = next(c for c in cases if O.V(bytearray(c[0].tobytes()), 0, O.ARENA_STATE).n_records > 0)
    t = rsx.v3_template(sd)
    b = bytearray(rsx.v3_write_arena(s, sd, t))
    cont = b.index(b"CONT") + 4
    n = struct.unpack_from("<I", b, cont)[0]
    rec_len = 1 + 4 + 4 + 60 + 12 + 4 + 1  # is_swap, two indices, one manifold point with applied_impulse and is_special
    first = cont + 4
    # repeat the last (stored) record until there are 17 stored ones
    v = O.V(bytearray(s.tobytes()), 0, O.ARENA_STATE)
    stored = v.n_records
    last = bytes(b[first + (n - 1) * rec_len:first + n * rec_len])
    extra = 17 - stored
    nb = bytes(b[:cont]) + struct.pack("<I", n + extra) + bytes(b[first:first + n * rec_len]) + last * extra + bytes(b[first + n * rec_len:])
    _both_refuse(rsx, nb, sd, "stored contact records over the cap")


def _full_static(rsx):
    """A StaticData of the synthetic world padded to the exact sizes the static importer requires (8,020 triangles
    and leaves, 3,754 BVH nodes, 1,210 static ray-cell entries): filler records appended to the last mesh and the last
    cell.  Only the format round trip uses it."""
    sd = rsx.build_static(7, 1, 5)
    v = O.V(bytearray(sd.tobytes()), 0, O.STATIC_DATA)
    m = v.meshes[15]
    tris = sum(v.meshes[k].tri_count for k in range(16))
    nodes = sum(v.meshes[k].node_count for k in range(16))
    leaves = sum(v.meshes[k].leaf_count for k in range(16))
    rng = np.random.default_rng(3)
    for i in range(tris, O.MAX_TRIS):
        v.tris[i].assign(rng.integers(0, 2**32, 12, dtype=np.uint32).tobytes())
        v.infos[i].assign(struct.pack("<I3I", int(rng.integers(0, 256)), *rng.integers(0, 2**32, 3, dtype=np.uint32)))
    for i in range(nodes, O.MAX_NODES):
        vals = rng.integers(0, 2**32, 30, dtype=np.uint32)
        vals[28] &= 0xFF
        v.nodes[i].assign(vals.tobytes())
    for i in range(leaves, O.MAX_LEAVES):
        v.leaves[i].assign(rng.integers(0, 2**32, 7, dtype=np.uint32).tobytes())
    m.tri_count = m.tri_count + O.MAX_TRIS - tris
    m.node_count = m.node_count + O.MAX_NODES - nodes
    m.leaf_count = m.leaf_count + O.MAX_LEAVES - leaves
    v.bodies[m.body].mesh_tri_count = m.tri_count
    entries = sum(v.cells[c].count for c in range(O.NUM_GRID_CELLS))
    last = v.cells[O.NUM_GRID_CELLS - 1]
    assert last.first + last.count == entries
    for i in range(entries, O.MAX_CELL_ENTRIES):
        v.cell_handles[i] = 1 + i % 20
    last.count = last.count + O.MAX_CELL_ENTRIES - entries
    for c in range(O.NUM_GRID_CELLS):  # an empty cell's range starts at 0 on import
        if v.cells[c].count == 0:
            v.cells[c].first = 0
    return np.frombuffer(bytes(v.b), np.uint32).copy()


def test_static_export_matches_oracle_and_imports_back(rsx):
    sd = _full_static(rsx)
    b = rsx.v3_write_static(sd)
    ref, cfg = O.write_static(sd)
    assert b == ref
    assert rsx.v3_config_hash(sd) == cfg
    assert b[:8] == b"V3STATIC" and struct.unpack_from("<IQQ", b, 8) == (3, O.fnv1a64(b[76:]), len(b) - 76)
    got = rsx.v3_parse_static(b)
    assert np.array_equal(got, sd), np.nonzero(got != sd)[0][:8]  # table_sin: the same correctly rounded generator
    pyw = O.parse_static(b)
    ts = O.STATIC_DATA.fields["table_sin"][0] // 4
    assert np.array_equal(pyw[:ts], sd[:ts])


def test_static_refusals_match_oracle(rsx):
    sd = _full_static(rsx)
    b = rsx.v3_write_static(sd)

    def both(data, msg):
        with pytest.raises(rsx.RsxError) as e:
            rsx.v3_parse_static(data)
        assert msg in str(e.value), str(e.value)
        with pytest.raises(O.DumpError) as e2:
            O.parse_static(data)
        assert str(e2.value) == msg
    both(b"V3STATIX" + b[8:], "not a static dump (magic)")
    both(b[:8] + struct.pack("<I", 2) + b[12:], "unsupported static dump version 2 (need 3: re-vendor V3)")
    both(b[:-1], "static dump payload length mismatch")
    flipped = bytearray(b)
    flipped[200] ^= 1
    both(bytes(flipped), "static dump payload hash mismatch")
    # the synthetic world as it is (fewer triangles than the importer's fixed size)
    small = rsx.v3_write_static(rsx.build_static(7, 0, 0))
    n = struct.unpack_from("<I", small, 28 + 12)[0]
    both(small, f"static dump count 3 is {n}; StaticData is sized for 8020 (the project's 16 Soccar meshes)")
