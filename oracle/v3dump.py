"""Test infrastructure: an independent CPU restatement of the V3 dump format, the oracle that the C ABI's V3 import and
export (rsx_v3_parse_arena / rsx_v3_write_arena / rsx_v3_parse_static / rsx_v3_write_static) are checked against.
Only tests import this file.

It follows the reference's crates/rocketsim-cuda/src/dump.rs (the importer and exporter of the Rust host crate, lines
cited per function) and the V3 side of the format in v3/rocketsim-dump.patch (src/dump.rs there, and the
export_static section order in rocketsim/src/sim/arena/base.rs of the patch).  The structures are described here from
the reference's own header (cuda/sim/arena_state.cuh:42-339), by field name, not from this project's headers, so an
error in either layout shows up as a difference.

Parity status: the reference's dump code is Rust and cannot be built in this image (no cargo), and the reference
checks in no dump files; this restatement is pinned by the format's fixed sizes (68-byte arena header, 76-byte
static header, 219-byte body records, the published FNV-1a 64 test vectors) and by agreeing byte for byte with the
C++ implementation, which was written separately from it.
"""
from __future__ import annotations

import struct

import numpy as np

# ---- layout types: every field is bytes at an offset; f32 fields are kept as their u32 bits ------------------------


class T:
    def __init__(self, kind, size, fmt=None, fields=None, elem=None, n=0):
        self.kind, self.size, self.fmt, self.fields, self.elem, self.n = kind, size, fmt, fields, elem, n


U32 = T("prim", 4, "I")
F32 = T("prim", 4, "I")  # bits
U16 = T("prim", 2, "H")


def st(*fields):
    offs, off = {}, 0
    for name, t in fields:
        offs[name] = (off, t)
        off += t.size
    return T("struct", off, fields=offs)


def arr(t, n):
    return T("arr", t.size * n, elem=t, n=n)


def opt(t):
    return st(("some", U32), ("v", t))


VEC3 = st(("x", F32), ("y", F32), ("z", F32))
MAT3 = st(("x_axis", VEC3), ("y_axis", VEC3), ("z_axis", VEC3))
AFF3 = st(("matrix3", MAT3), ("translation", VEC3))
QUAT = st(("x", F32), ("y", F32), ("z", F32), ("w", F32))
AABB = st(("min", VEC3), ("max", VEC3))
U64 = st(("lo", U32), ("hi", U32))

NUM_BODIES, NUM_DYN, NUM_CARS, NUM_WHEELS, NUM_PADS, NUM_HANDLES, NUM_MESHES, NUM_PLANES = 23, 3, 2, 4, 34, 24, 16, 4
NUM_EDGES = 2 * NUM_HANDLES
MAX_MANIFOLDS, MAX_POINTS, MAX_ACTIVE, MAX_RECORDS, MAX_PAIRS, MAX_DYN_CELLS = 16, 4, 16, 16, 16, 64
MAX_TRIS, MAX_NODES, MAX_LEAVES, TABLE_SIN_LEN, NUM_GRID_CELLS, MAX_CELL_ENTRIES, NUM_MUT = 8020, 3754, 8020, 16384, 242, 1210, 20
OVF_MANIFOLDS, OVF_ACTIVE, OVF_RECORDS, OVF_PAIRS, OVF_DYN_CELLS = 0, 1, 2, 3, 4
EV_CAR_HIT_WORLD, EV_BALL_HIT_WORLD, EV_BALL_WALL = 10, 12, 14
UI_NONE, UI_CAR, UI_BALL = 0, 1, 2

CONTROLS = st(*[(k, F32) for k in ("throttle", "steer", "pitch", "yaw", "roll")], ("jump", U32), ("boost", U32), ("handbrake", U32))
HIT_INFO = st(("hit_point", VEC3), ("hit_normal", VEC3), ("hit_fraction", F32), ("user_info", U32))
RAYCAST_INFO = st(("contact_normal", VEC3), ("contact_point", VEC3), ("ground_body_idx", U32), ("suspension_length", F32),
                  ("impulse", VEC3), ("ground_stick", opt(VEC3)), ("is_in_contact_with_world", U32),
                  ("clipped_inv_contact_dot_suspension", F32), ("suspension_relative_vel", F32))
WHEEL = st(("raycast_info", opt(RAYCAST_INFO)), ("hard_point", VEC3), ("axle_dir", VEC3), ("engine_force", F32), ("brake", F32),
           ("steer_angle", F32), ("vel_at_contact_point", VEC3), ("lat_friction", F32), ("long_friction", F32), ("extra_pushback", F32))
CAR = st(("dodge_deadzone", F32), ("vel_impulse_cache", VEC3), ("sticky_gate_prev", U32), ("pos", VEC3), ("rot_mat", MAT3),
         ("vel", VEC3), ("ang_vel", VEC3), ("controls", CONTROLS), ("has_jumped", U32), ("has_double_jumped", U32),
         ("has_flipped", U32), ("flip_rel_torque", VEC3), ("jump_ticks", U32), ("flip_time", F32), ("is_flipping", U32),
         ("is_jumping", U32), ("jump_hold_broken", U32), ("air_time", F32), ("air_time_since_jump", F32), ("boost", F32),
         ("handbrake_val", F32), ("is_supersonic", U32), ("supersonic_grace_timer", F32), ("time_since_boosted", F32),
         ("boosting_time", F32), ("is_boosting", U32), ("is_auto_flipping", U32), ("auto_flip_timer", F32),
         ("auto_flip_torque_scale", F32), ("bump_cooldown_timer", F32), ("bump_cooldown_victim", opt(U32)),
         ("last_extra_hit_tick", opt(U64)), ("is_demoed", U32), ("demo_respawn_timer", F32), ("is_on_ground", U32),
         ("wheels_with_contact", arr(opt(HIT_INFO), NUM_WHEELS)), ("world_contact_normal", opt(VEC3)),
         ("prev_controls", CONTROLS), ("wheels", arr(WHEEL, NUM_WHEELS)))
PAD_TOUCHING = st(("n", U32), ("car_idx", arr(U32, NUM_CARS)))
BALL_DYN = st(("pos", VEC3), ("rot_mat", MAT3), ("vel", VEC3), ("ang_vel", VEC3), ("tick_count_since_kickoff", U64))
BODY = st(("collision_flags", U32), ("activation", U32), ("deactivation_time", F32), ("world_trans", AFF3), ("world_quat", QUAT),
          ("interp_world_trans", AFF3), ("lin_vel", VEC3), ("ang_vel", VEC3), ("inv_inertia_tensor_world", MAT3),
          ("accum_lin_vel", VEC3), ("accum_ang_vel", VEC3), ("cached_linear_damping", F32), ("cached_damping_time_step", F32),
          ("cached_linear_damping_value", F32))
MANIFOLD_POINT = st(("local_point_a", VEC3), ("local_point_b", VEC3), ("pos_world_on_b", VEC3), ("pos_world_on_a", VEC3),
                    ("normal_world_on_b", VEC3), ("distance_1", F32), ("combined_friction", F32), ("combined_restitution", F32),
                    ("is_special", U32))
MANIFOLD = st(("body0_idx", U32), ("body1_idx", U32), ("point_count", U32), ("points", arr(MANIFOLD_POINT, MAX_POINTS)))
RECORD_POINT = st(("pos_world_on_b", VEC3), ("pos_world_on_a", VEC3), ("normal_world_on_b", VEC3))
CONTACT_RECORD = st(("is_swap", U32), ("rb_idx_a", U32), ("rb_idx_b", U32), ("point", RECORD_POINT))
DYN_PROXY = st(("aabb", AABB), ("cell_idx", U32), ("indices", arr(U32, 3)))
HANDLE_EDGES = st(("min", arr(U16, 3)), ("max", arr(U16, 3)))
EDGE = st(("pos", U16), ("handle", U16))
DYN_CELL = st(("cell", U32), ("handle", U32))
PAIR = st(("proxy0", U32), ("proxy1", U32))
ARENA_STATE = st(("tick_count", U64), ("rng", U64), ("ball", BALL_DYN), ("cars", arr(CAR, NUM_CARS)),
                 ("pad_gave_boost", arr(opt(U64), NUM_PADS)), ("pad_touching", arr(PAD_TOUCHING, NUM_PADS)),
                 ("bodies", arr(BODY, NUM_DYN)), ("n_manifolds", U32), ("manifolds", arr(MANIFOLD, MAX_MANIFOLDS)),
                 ("n_dyn_cells", U32), ("dyn_cells", arr(DYN_CELL, MAX_DYN_CELLS)), ("dyn_proxy", arr(DYN_PROXY, NUM_DYN)),
                 ("handle_edges", arr(HANDLE_EDGES, NUM_HANDLES)), ("edges", arr(arr(EDGE, NUM_EDGES), 3)), ("n_pairs", U32),
                 ("pairs", arr(PAIR, MAX_PAIRS)), ("overflow", arr(U32, 6)), ("events", U32), ("n_active", U32),
                 ("active", arr(U32, MAX_ACTIVE)), ("fold_events", U32), ("fold_car_normal", arr(VEC3, NUM_CARS)),
                 ("n_records", U32), ("records", arr(CONTACT_RECORD, MAX_RECORDS)))

MESH_INFO = st(*[(k, U32) for k in ("body", "tri_first", "tri_count", "node_first", "node_count", "leaf_first", "leaf_count")],
               ("aabb_ident_cache", AABB), ("root_aabb", AABB))
TRI = st(("p0", VEC3), ("p1", VEC3), ("p2", VEC3), ("normal", VEC3))
WIDE_NODE = st(*[(k, arr(F32, 4)) for k in ("min_x", "min_y", "min_z", "max_x", "max_y", "max_z")], ("children", arr(U32, 4)),
               ("child_count", U32), ("valid_mask", U32))
LEAF = st(("bounds", AABB), ("leaf_idx", U32))
TRI_INFO = st(("flags", U32), ("edge_v0_v1_angle", F32), ("edge_v1_v2_angle", F32), ("edge_v2_v0_angle", F32))
PLANE = st(("body", U32), ("plane_normal", VEC3), ("is_single_axis", U32), ("single_axis_idx", U32), ("single_axis_backwards", U32),
           ("aabb_ident_cache", AABB), ("aabb_cache", AABB))
BODY_CONST = st(*[(k, U32) for k in ("world_array_idx", "user_idx", "user_pointer", "broadphase_handle", "filter_group", "filter_mask")],
                ("mass", F32), ("inv_mass", F32), ("inv_inertia_local", VEC3), ("inv_mass_splat", VEC3), ("friction", F32),
                ("restitution", F32), ("contact_processing_threshold", F32), ("contact_breaking_threshold", F32),
                ("linear_damping", F32), ("linear_sleeping_threshold", F32), ("angular_sleeping_threshold", F32), ("pose", AFF3),
                ("shape_kind", U32), ("sphere_implicit_dim", VEC3), ("sphere_margin", F32), ("box_half_extents", VEC3),
                ("box_margin", F32), ("child_trans", AFF3), ("compound_local_aabb", AABB), ("mesh_tri_count", U32))
WHEEL_CONST = st(("chassis_connection_point_cs", VEC3), ("suspension_rest_length_1", F32), ("wheels_radius", F32),
                 ("suspension_force_scale", F32), ("real_ray_length", F32))
CAR_CONST = st(("car_idx", U32), ("team", U32), ("rigid_body_idx", U32), ("three_wheels", U32), ("hitbox_size", VEC3),
               ("hitbox_pos_offset", VEC3), ("wheels", arr(WHEEL_CONST, NUM_WHEELS)))
PAD_CONST = st(("pos", VEC3), ("is_big", U32), ("box_radius", F32), ("cyl_radius", F32), ("max_cooldown", F32), ("boost_amount", F32),
               ("aabb", AABB))
PROXY_CONST = st(("client_obj_idx", U32), ("filter_group", U32), ("filter_mask", U32), ("unique_id", U32), ("aabb", AABB),
                 ("cell_idx", U32), ("indices", arr(U32, 3)))
CELL_RANGE = st(("first", U32), ("count", U32))
STATIC_DATA = st(("game_mode", U32), ("no_ball_rot", U32), ("ball_body", U32), ("gravity_uu", VEC3), ("mut_f", arr(F32, NUM_MUT)),
                 ("unlimited_flips", U32), ("unlimited_double_jumps", U32), ("recharge_boost_enabled", U32),
                 ("recharge_boost_per_second", F32), ("recharge_boost_delay", F32), ("demo_mode", U32), ("enable_team_demos", U32),
                 ("goal_base_threshold_y", F32), ("boost_pads_enabled", U32), ("gravity_bt", VEC3), ("dyn_body", arr(U32, NUM_DYN)),
                 ("grid_min_pos", VEC3), ("grid_max_pos", VEC3), ("grid_cell_size", F32), ("grid_cell_size_sq", F32),
                 ("grid_num_cells", arr(U32, 3)), ("sap_world_aabb_min", VEC3), ("sap_quantize", VEC3), ("sap_handle_mask", U32),
                 ("sap_sentinel", U32), ("sap_max_handles", U32), ("sap_world_half_extent", F32), ("max_pad_z", F32),
                 ("dyn_handle", arr(U32, NUM_DYN)), ("bodies", arr(BODY_CONST, NUM_BODIES)), ("planes", arr(PLANE, NUM_PLANES)),
                 ("meshes", arr(MESH_INFO, NUM_MESHES)), ("cars", arr(CAR_CONST, NUM_CARS)), ("pads", arr(PAD_CONST, NUM_PADS)),
                 ("proxies", arr(PROXY_CONST, NUM_HANDLES)), ("cells", arr(CELL_RANGE, NUM_GRID_CELLS)),
                 ("cell_handles", arr(U32, MAX_CELL_ENTRIES)), ("infos", arr(TRI_INFO, MAX_TRIS)), ("tris", arr(TRI, MAX_TRIS)),
                 ("nodes", arr(WIDE_NODE, MAX_NODES)), ("leaves", arr(LEAF, MAX_LEAVES)), ("table_sin", arr(F32, TABLE_SIN_LEN)))
ARENA_WORDS = ARENA_STATE.size // 4
TICK_WORDS = ARENA_STATE.fields["n_active"][0] // 4
STATIC_WORDS = STATIC_DATA.size // 4


class V:
    """A view of one structure or array inside a bytearray."""
    __slots__ = ("b", "o", "t")

    def __init__(self, b, o, t):
        object.__setattr__(self, "b", b)
        object.__setattr__(self, "o", o)
        object.__setattr__(self, "t", t)

    def _at(self, key):
        if isinstance(key, str):
            off, t = self.t.fields[key]
        else:
            if not 0 <= key < self.t.n:
                raise IndexError(key)
            off, t = key * self.t.elem.size, self.t.elem
        return self.o + off, t

    def get(self, key):
        o, t = self._at(key)
        return struct.unpack_from("<" + t.fmt, self.b, o)[0] if t.kind == "prim" else V(self.b, o, t)

    def set(self, key, v):
        o, t = self._at(key)
        struct.pack_into("<" + t.fmt, self.b, o, v)

    __getattr__ = get
    __getitem__ = get
    __setitem__ = set

    def __setattr__(self, key, v):
        self.set(key, v)

    def raw(self) -> bytes:
        return bytes(self.b[self.o:self.o + self.t.size])

    def assign(self, data: bytes):
        self.b[self.o:self.o + self.t.size] = data


def f32(bits: int) -> float:
    return struct.unpack("<f", struct.pack("<I", bits))[0]


def f32_bits(x: float) -> int:
    return struct.unpack("<I", struct.pack("<f", x))[0]


class DumpError(Exception):
    pass


def fnv1a64(data: bytes) -> int:
    """dump.rs:29-36: FNV-1a 64."""
    h = 0xCBF29CE484222325
    for c in data:
        h = ((h ^ c) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
    return h


# ---- the byte stream in both directions (dump.rs:39-207) ----------------------------------------------------------
class Wr:
    READ = False

    def __init__(self):
        self.out = bytearray()
        self.err = None
        self.marks = []

    def fail(self, msg):
        if self.err is None:
            self.err = msg

    def prim(self, fmt, v, k):
        self.out += struct.pack("<" + fmt, v.get(k))

    def u8(self, v, k):
        self.out.append(v.get(k) & 0xFF)

    def u8v(self, x):  # a u8 that is not a state field; returns the value
        self.out.append(x & 0xFF)
        return x

    def u16v(self, x):
        self.out += struct.pack("<H", x)
        return x

    def u32v(self, x):
        self.out += struct.pack("<I", x)
        return x

    def u64v(self, x):
        self.out += struct.pack("<Q", x)
        return x

    def rawv(self, data: bytes):
        self.out += data
        return data

    def count(self, n):
        self.out += struct.pack("<I", n)
        return n

    def mark(self):
        self.marks.append(len(self.out))


class Rd:
    READ = True

    def __init__(self, data: bytes):
        self.b = data
        self.p = 0
        self.err = None

    def remaining(self):
        return len(self.b) - self.p

    def fail(self, msg):
        if self.err is None:
            self.err = msg

    def _take(self, n):
        if self.remaining() < n:
            self.fail("dump truncated")
            self.p = len(self.b)
            return bytes(n)
        out = self.b[self.p:self.p + n]
        self.p += n
        return out

    def prim(self, fmt, v, k):
        v.set(k, struct.unpack("<" + fmt, self._take(struct.calcsize("<" + fmt)))[0])

    def u8(self, v, k):
        v.set(k, self._take(1)[0])

    def u8v(self, _x):
        return self._take(1)[0]

    def u16v(self, _x):
        return struct.unpack("<H", self._take(2))[0]

    def u32v(self, _x):
        return struct.unpack("<I", self._take(4))[0]

    def u64v(self, _x):
        return struct.unpack("<Q", self._take(8))[0]

    def rawv(self, data: bytes):
        if self.remaining() < len(data):
            self.fail("dump truncated")
            self.p = len(self.b)
            return data
        out = bytes(self.b[self.p:self.p + len(data)])
        self.p += len(data)
        return out

    def count(self, _n):
        x = self.u32v(0)
        if x > self.remaining():
            self.fail("count exceeds the bytes left")
            return 0
        return x

    def mark(self):
        pass


def u32(io, v, k):
    io.prim("I", v, k)


def u16(io, v, k):
    io.prim("H", v, k)


def flag(io, v, k):
    """A V3 bool as one byte held as a u32 (dump.rs:58-63)."""
    if io.READ:
        io.u8(v, k)
    else:
        io.u8v(1 if v.get(k) != 0 else 0)


def byte(io, v, k):
    io.u8(v, k)


def tag(io, t: bytes):
    io.mark()
    want = struct.unpack("<I", t)[0]
    if io.u32v(want) != want:
        io.fail(f"section tag {t.decode()} expected")


def vec3(io, v):
    for k in ("x", "y", "z"):
        u32(io, v, k)


def mat3(io, m):
    for k in ("x_axis", "y_axis", "z_axis"):
        vec3(io, m.get(k))


def aff3(io, a):
    mat3(io, a.matrix3)
    vec3(io, a.translation)


def quat(io, q):
    for k in ("x", "y", "z", "w"):
        u32(io, q, k)


def aabb(io, a):
    vec3(io, a.get("min"))
    vec3(io, a.get("max"))


def u64s(io, v):
    x = io.u64v(v.lo | v.hi << 32)
    v.lo, v.hi = x & 0xFFFFFFFF, x >> 32


def opt_with(io, o, f):
    flag(io, o, "some")
    f(io, o.v)


def opt_idx(io, o):
    flag(io, o, "some")
    u32(io, o, "v")


# ---- the arena (dump.rs:241-848) ----------------------------------------------------------------------------------
def io_controls(io, c):
    for k in ("throttle", "steer", "pitch", "yaw", "roll"):
        u32(io, c, k)
    for k in ("jump", "boost", "handbrake"):
        flag(io, c, k)


def io_hit(io, h):
    vec3(io, h.hit_point)
    vec3(io, h.hit_normal)
    u32(io, h, "hit_fraction")
    byte(io, h, "user_info")


def io_point(io, p):
    for k in ("local_point_a", "local_point_b", "pos_world_on_b", "pos_world_on_a", "normal_world_on_b"):
        vec3(io, p.get(k))
    for k in ("distance_1", "combined_friction", "combined_restitution"):
        u32(io, p, k)
    if io.u32v(0) != 0 and io.READ:  # applied_impulse: always 0 in V3's dumps, not state
        io.fail("manifold point with a non-zero applied_impulse")
    flag(io, p, "is_special")


def io_raycast(io, r):
    vec3(io, r.contact_normal)
    vec3(io, r.contact_point)
    u32(io, r, "ground_body_idx")
    u32(io, r, "suspension_length")
    vec3(io, r.impulse)
    opt_with(io, r.ground_stick, vec3)
    flag(io, r, "is_in_contact_with_world")
    u32(io, r, "clipped_inv_contact_dot_suspension")
    u32(io, r, "suspension_relative_vel")


def io_wheel(io, w):
    opt_with(io, w.raycast_info, io_raycast)
    vec3(io, w.hard_point)
    vec3(io, w.axle_dir)
    for k in ("engine_force", "brake", "steer_angle"):
        u32(io, w, k)
    vec3(io, w.vel_at_contact_point)
    for k in ("lat_friction", "long_friction", "extra_pushback"):
        u32(io, w, k)


def io_car(io, c):
    u32(io, c, "dodge_deadzone")
    vec3(io, c.vel_impulse_cache)
    flag(io, c, "sticky_gate_prev")
    vec3(io, c.pos)
    mat3(io, c.rot_mat)
    vec3(io, c.vel)
    vec3(io, c.ang_vel)
    io_controls(io, c.controls)
    for k in ("has_jumped", "has_double_jumped", "has_flipped"):
        flag(io, c, k)
    vec3(io, c.flip_rel_torque)
    u32(io, c, "jump_ticks")
    u32(io, c, "flip_time")
    for k in ("is_flipping", "is_jumping", "jump_hold_broken"):
        flag(io, c, k)
    for k in ("air_time", "air_time_since_jump", "boost", "handbrake_val"):
        u32(io, c, k)
    flag(io, c, "is_supersonic")
    for k in ("supersonic_grace_timer", "time_since_boosted", "boosting_time"):
        u32(io, c, k)
    flag(io, c, "is_boosting")
    flag(io, c, "is_auto_flipping")
    for k in ("auto_flip_timer", "auto_flip_torque_scale", "bump_cooldown_timer"):
        u32(io, c, k)
    opt_idx(io, c.bump_cooldown_victim)
    opt_with(io, c.last_extra_hit_tick, u64s)
    flag(io, c, "is_demoed")
    u32(io, c, "demo_respawn_timer")
    flag(io, c, "is_on_ground")
    for w in range(NUM_WHEELS):
        opt_with(io, c.wheels_with_contact[w], io_hit)
    opt_with(io, c.world_contact_normal, vec3)
    io_controls(io, c.prev_controls)
    for w in range(NUM_WHEELS):
        io_wheel(io, c.wheels[w])


def io_body(io, b):
    """One dynamic BODY record (219 bytes); companion_id is written as none and ignored on read."""
    byte(io, b, "collision_flags")
    io.u8v(0)
    io.u32v(0)
    byte(io, b, "activation")
    aff3(io, b.world_trans)
    quat(io, b.world_quat)
    aff3(io, b.interp_world_trans)
    u32(io, b, "deactivation_time")
    vec3(io, b.lin_vel)
    vec3(io, b.ang_vel)
    mat3(io, b.inv_inertia_tensor_world)
    vec3(io, b.accum_lin_vel)
    vec3(io, b.accum_ang_vel)
    for k in ("cached_linear_damping", "cached_damping_time_step", "cached_linear_damping_value"):
        u32(io, b, k)


def table_index(a, b):
    lo, hi = min(a, b), max(a, b)
    return hi * (hi + 1) // 2 + lo


def fold_records(s, sd, recs):
    """dump.rs:387-422."""
    s.fold_events = 0
    for c in range(NUM_CARS):
        s.fold_car_normal[c].assign(bytes(12))
    s.n_records = 0
    s.records.assign(bytes(CONTACT_RECORD.size * MAX_RECORDS))
    for r in recs:
        if r["a"] >= NUM_BODIES or r["b"] >= NUM_BODIES:
            raise DumpError("contact record body index out of range")
        a, b = sd.bodies[r["a"]], sd.bodies[r["b"]]
        if a.user_idx == UI_CAR and b.user_idx in (UI_BALL, UI_CAR):
            if s.n_records >= MAX_RECORDS:
                raise DumpError("stored contact records over the cap")
            d = s.records[s.n_records]
            d.is_swap, d.rb_idx_a, d.rb_idx_b = r["swap"], r["a"], r["b"]
            d.point.assign(r["point"])
            s.n_records = s.n_records + 1
        elif a.user_idx == UI_CAR:
            car = a.user_pointer
            if car >= NUM_CARS:
                raise DumpError("contact record of a car index outside the arena")
            s.fold_events = s.fold_events | 1 << (EV_CAR_HIT_WORLD + car)
            s.fold_car_normal[car].assign(r["point"][24:36])
        elif a.user_idx == UI_BALL and b.user_idx == UI_NONE:
            s.fold_events = s.fold_events | 1 << EV_BALL_HIT_WORLD
            if abs(f32(struct.unpack_from("<I", r["point"], 32)[0])) < 0.8:
                s.fold_events = s.fold_events | 1 << EV_BALL_WALL


def unfold_records(s, sd):
    """dump.rs:424-447."""
    world = next(i for i in range(NUM_BODIES) if sd.bodies[i].user_idx == UI_NONE)

    def rec(a, normal_bytes):
        return {"swap": 0, "a": a, "b": world, "point": bytes(24) + normal_bytes}
    out = []
    fe = s.fold_events
    if fe >> EV_BALL_HIT_WORLD & 1:
        n = (1.0, 0.0, 0.0) if fe >> EV_BALL_WALL & 1 else (0.0, 0.0, 1.0)
        out.append(rec(sd.dyn_body[0], struct.pack("<3f", *n)))
    for car in range(NUM_CARS):
        if fe >> (EV_CAR_HIT_WORLD + car) & 1:
            out.append(rec(sd.dyn_body[1 + car], s.fold_car_normal[car].raw()))
    for i in range(s.n_records):
        r = s.records[i]
        out.append({"swap": r.is_swap, "a": r.rb_idx_a, "b": r.rb_idx_b, "point": r.point.raw()})
    return out


def empty_template():
    return {"config_hash": 0, "static_body": [bytes(219)] * NUM_BODIES, "num_handles": 0, "next_new_handle": 0,
            "manifold_stride": 0, "ball_other": bytes(24), "ball_other_set": False}


def io_arena(io, s, sd, t):
    """dump.rs:449-848; raises DumpError with the reference's message."""
    R = io.READ

    def check():
        if io.err is not None:
            raise DumpError(io.err)
    tag(io, b"ARNA")
    u64s(io, s.tick_count)
    u64s(io, s.rng)
    if io.u8v(0) != 0 and R:
        io.fail("a ball-only arena")
    tag(io, b"BALL")
    vec3(io, s.ball.pos)
    mat3(io, s.ball.rot_mat)
    vec3(io, s.ball.vel)
    vec3(io, s.ball.ang_vel)
    other = io.rawv(t["ball_other"])
    if R:
        if not t["ball_other_set"]:
            t["ball_other"], t["ball_other_set"] = other, True
        elif other != t["ball_other"]:
            io.fail("Heatseeker or Dropshot ball info changed between dumps")
    u64s(io, s.ball.tick_count_since_kickoff)
    if io.u8v(0) != 0 and R:
        io.fail("Snowday ground_stick_applied is set")
    tag(io, b"CARS")
    if io.count(NUM_CARS) != NUM_CARS:
        io.fail("not a 2-car arena")
        check()
    for c in range(NUM_CARS):
        io_car(io, s.cars[c])
    tag(io, b"PADS")
    if io.count(NUM_PADS) != NUM_PADS:
        io.fail("not a 34-pad arena")
        check()
    for p in range(NUM_PADS):
        opt_with(io, s.pad_gave_boost[p], u64s)
        pt = s.pad_touching[p]
        n = io.count(pt.n)
        if n > NUM_CARS:
            io.fail("a pad touched by more cars than the arena has")
            check()
        pt.n = n
        for k in range(n):
            u32(io, pt.car_idx, k)
    tag(io, b"CONT")
    recs = [] if R else unfold_records(s, sd)
    n = io.count(len(recs))
    if R:
        recs = [{"swap": 0, "a": 0, "b": 0, "point": bytes(36)} for _ in range(n)]
    scratch = V(bytearray(MANIFOLD_POINT.size + 4), 0, MANIFOLD_POINT)
    for r in recs:
        swap = V(bytearray(4), 0, st(("x", U32)))
        swap.x = r["swap"]
        flag(io, swap, "x")
        r["swap"] = swap.x
        r["a"] = io.u32v(r["a"])
        r["b"] = io.u32v(r["b"])
        scratch.assign(bytes(MANIFOLD_POINT.size))
        scratch.b[24:60] = r["point"]  # pos_world_on_b, pos_world_on_a, normal_world_on_b
        io_point(io, scratch)
        r["point"] = bytes(scratch.b[24:60])
    if R and io.err is None:
        try:
            fold_records(s, sd, recs)
        except DumpError as e:
            s.overflow[OVF_RECORDS] = s.overflow[OVF_RECORDS] + 1
            io.fail(str(e))
            check()
    if io.count(0) != 0:
        io.fail("ball-world contact records present")
        check()
    io.u8v(0)
    tag(io, b"BODY")
    if io.count(NUM_BODIES) != NUM_BODIES:
        io.fail("not a 23-body arena")
        check()
    dyn_body = [sd.dyn_body[d] for d in range(NUM_DYN)]
    for i in range(NUM_BODIES):
        if i in dyn_body:
            io_body(io, s.bodies[dyn_body.index(i)])
        elif R:
            rec = bytearray(io.rawv(bytes(219)))
            rec[1:6] = bytes(5)
            if t["static_body"][i] == bytes(219):
                t["static_body"][i] = bytes(rec)
        else:
            io.rawv(t["static_body"][i])
    tag(io, b"DISP")
    nm = io.count(s.n_manifolds)
    if R:
        if nm > MAX_MANIFOLDS:
            s.overflow[OVF_MANIFOLDS] = s.overflow[OVF_MANIFOLDS] + 1
            io.fail("retained manifolds over the cap")
            check()
        s.n_manifolds = nm
    for i in range(nm):
        m = s.manifolds[i]
        u32(io, m, "body0_idx")
        u32(io, m, "body1_idx")
        b0, b1 = m.body0_idx, m.body1_idx
        key = min(b0, b1) << 32 | max(b0, b1)
        if io.u64v(key) != key and R:
            io.fail("manifold pair_key is not min << 32 | max")
        if b0 >= NUM_BODIES or b1 >= NUM_BODIES:
            io.fail("manifold body index out of range")
            check()
        cbt = min(f32(sd.bodies[b0].contact_breaking_threshold), f32(sd.bodies[b1].contact_breaking_threshold))
        cpt = min(f32(sd.bodies[b0].contact_processing_threshold), f32(sd.bodies[b1].contact_processing_threshold))
        got_cbt = io.u32v(f32_bits(cbt))
        got_cpt = io.u32v(f32_bits(cpt))
        if R and (got_cbt != f32_bits(cbt) or got_cpt != f32_bits(cpt)):
            io.fail("a manifold threshold is not the min over its two bodies")
            check()
        u32(io, m, "point_count")
        if m.point_count > MAX_POINTS:
            io.fail("manifold with more than 4 points")
            check()
        for k in range(MAX_POINTS):
            io_point(io, m.points[k])
    na = io.count(s.n_active)
    if R:
        if na > MAX_ACTIVE:
            s.overflow[OVF_ACTIVE] = s.overflow[OVF_ACTIVE] + 1
            io.fail("active manifolds over the cap")
            check()
        s.n_active = na
    for i in range(na):
        u32(io, s.active, i)
    stride = io.u32v(t["manifold_stride"] if R else (32 if nm > 0 else t["manifold_stride"]))
    tl = io.count(stride * stride)
    if R:
        t["manifold_stride"] = stride
        if tl != stride * stride:
            io.fail("manifold table length is not stride squared")
            check()
    table = [0] * tl
    for i in range(nm):
        m = s.manifolds[i]
        lo, hi = min(m.body0_idx, m.body1_idx), max(m.body0_idx, m.body1_idx)
        if hi >= stride:
            io.fail("manifold body index outside the table")
            check()
        table[lo * stride + hi] = i + 1
    for e in table:
        if io.u32v(e) != e and R:
            io.fail("manifold table is not the search of the pool")
            check()
    tag(io, b"BROA")
    if R:
        entries, last = [], None
        for _ in range(io.count(0)):
            cell = io.u32v(0)
            if last is not None and last >= cell:
                io.fail("dynamic ray cells not ascending")
                check()
            last = cell
            for _ in range(io.count(0)):
                entries.append((cell, io.u32v(0)))
            if io.err is not None:
                break
        if len(entries) > MAX_DYN_CELLS:
            s.overflow[OVF_DYN_CELLS] = s.overflow[OVF_DYN_CELLS] + 1
            io.fail("dynamic ray-cell entries over the cap")
            check()
        s.n_dyn_cells = len(entries)
        for k, (c, h) in enumerate(entries):
            s.dyn_cells[k].cell, s.dyn_cells[k].handle = c, h
    else:
        groups = []
        for k in range(s.n_dyn_cells):
            e = s.dyn_cells[k]
            if groups and groups[-1][0] == e.cell:
                groups[-1][1].append(e.handle)
            else:
                groups.append((e.cell, [e.handle]))
        io.count(len(groups))
        for c, hs in groups:
            io.u32v(c)
            io.count(len(hs))
            for h in hs:
                io.u32v(h)
    if io.count(NUM_HANDLES) != NUM_HANDLES:
        io.fail("not a 24-handle broadphase")
        check()
    dyn_handle = [sd.dyn_handle[d] for d in range(NUM_DYN)]
    for h in range(NUM_HANDLES):
        c = sd.proxies[h]
        obj = io.u32v(c.client_obj_idx)
        g = io.u8v(c.filter_group & 0xFF)
        m = io.u8v(c.filter_mask & 0xFF)
        uid = io.u32v(c.unique_id)
        if h in dyn_handle:
            dp = s.dyn_proxy[dyn_handle.index(h)]
            aabb(io, dp.aabb)
            u32(io, dp, "cell_idx")
            for k in range(3):
                u32(io, dp.indices, k)
        else:
            tmp = V(bytearray(c.raw()), 0, PROXY_CONST)
            aabb(io, tmp.aabb)
            u32(io, tmp, "cell_idx")
            for k in range(3):
                u32(io, tmp.indices, k)
            box_t = [f32(x) for x in struct.unpack("<6I", tmp.aabb.raw())]
            box_c = [f32(x) for x in struct.unpack("<6I", c.aabb.raw())]
            same = box_t == box_c and tmp.cell_idx == c.cell_idx and tmp.indices.raw() == c.indices.raw()
            if R and not same:
                io.fail("a static broadphase proxy differs from StaticData.proxies")
                check()
        if R and (obj != c.client_obj_idx or g != c.filter_group or m != c.filter_mask or uid != c.unique_id):
            io.fail("a broadphase proxy constant differs from StaticData.proxies")
            check()
    if io.count(NUM_HANDLES) != NUM_HANDLES:
        io.fail("handle_edges length")
        check()
    for h in range(NUM_HANDLES):
        e = s.handle_edges[h]
        for k in range(3):
            u16(io, e.get("min"), k)
        for k in range(3):
            u16(io, e.get("max"), k)
    for axis in range(3):
        if io.count(NUM_EDGES) != NUM_EDGES:
            io.fail("edge array length")
            check()
        for k in range(NUM_EDGES):
            u16(io, s.edges[axis][k], "pos")
            u16(io, s.edges[axis][k], "handle")
    t["num_handles"] = io.u16v(t["num_handles"])
    if io.count(0) != 0:
        io.fail("free_list is not empty")
        check()
    t["next_new_handle"] = io.u16v(t["next_new_handle"])
    np_ = io.count(s.n_pairs)
    if R:
        if np_ > MAX_PAIRS:
            s.overflow[OVF_PAIRS] = s.overflow[OVF_PAIRS] + 1
            io.fail("retained pairs over the cap")
            check()
        s.n_pairs = np_
    for i in range(np_):
        u32(io, s.pairs[i], "proxy0")
        u32(io, s.pairs[i], "proxy1")
    want = [(table_index(s.pairs[i].proxy0, s.pairs[i].proxy1), i + 1) for i in range(np_)]
    if R:
        got = [io.u32v(0) for _ in range(io.count(0))]
        seen = 0
        for i, g in enumerate(got):
            if g:
                seen += 1
                if (i, g) not in want:
                    io.fail("pair index table is not the search of the pair array")
                    check()
        if seen != np_:
            io.fail("pair index table and pair array disagree")
            check()
    else:
        n = max((i + 1 for i, _ in want), default=0)
        io.count(n)
        tbl = [0] * n
        for i, v in want:
            tbl[i] = v
        for v in tbl:
            io.u32v(v)
    check()


def io_island(io):
    """dump.rs:851-866."""
    tag(io, b"ISLD")
    for width in (4, 4, 8, 8, 4, 4):
        n = io.count(0)
        if io.READ and n:
            io.rawv(bytes(n * width))
    io.u8v(0)
    if io.err is not None:
        raise DumpError(io.err)


def parse_arena(data: bytes, sd_words: np.ndarray):
    """dump.rs:870-900: (state words, template)."""
    if len(data) < 68 or data[:8] != b"V3ARENA\0":
        raise DumpError("not an arena dump (magic)")
    version = struct.unpack_from("<I", data, 8)[0]
    if version != 2:
        raise DumpError(f"unsupported arena dump version {version}")
    sd = V(bytearray(np.ascontiguousarray(sd_words, np.uint32).tobytes()), 0, STATIC_DATA)
    s = V(bytearray(ARENA_STATE.size), 0, ARENA_STATE)
    t = empty_template()
    t["config_hash"] = struct.unpack_from("<Q", data, 12)[0]
    r = Rd(bytes(data[68:]))
    io_arena(r, s, sd, t)
    io_island(r)
    if r.remaining():
        raise DumpError(f"{r.remaining()} trailing bytes")
    return np.frombuffer(bytes(s.b), np.uint32).copy(), t


def write_arena(state_words: np.ndarray, sd_words: np.ndarray, t: dict) -> bytes:
    """dump.rs:902-944."""
    sd = V(bytearray(np.ascontiguousarray(sd_words, np.uint32).tobytes()), 0, STATIC_DATA)
    s = V(bytearray(np.ascontiguousarray(state_words, np.uint32).tobytes()), 0, ARENA_STATE)
    t = dict(t)
    w = Wr()
    io_arena(w, s, sd, t)
    io_island(w)
    nm = s.n_manifolds
    points = sum(s.manifolds[i].point_count for i in range(nm))
    stride = 32 if nm > 0 else t["manifold_stride"]
    counts = [NUM_BODIES, nm, s.n_active, points, stride * stride, NUM_HANDLES, s.n_pairs, s.n_dyn_cells, NUM_CARS, NUM_PADS,
              len(unfold_records(s, sd)), 0]
    return b"V3ARENA\0" + struct.pack("<IQ12I", 2, t["config_hash"], *counts) + bytes(w.out)


# ---- the static data (dump.rs:947-1300) ----------------------------------------------------------------------------
def io_static(io, sd):
    R = io.READ

    def expect(got, want, what):
        if got != want:
            io.fail(f"{what}: {got}, StaticData holds {want}")
            raise DumpError(io.err)
    tag(io, b"WRLD")
    byte(io, sd, "game_mode")
    flag(io, sd, "no_ball_rot")
    u32(io, sd, "ball_body")
    vec3(io, sd.gravity_uu)
    for k in range(NUM_MUT):
        u32(io, sd.mut_f, k)
    for k in ("unlimited_flips", "unlimited_double_jumps", "recharge_boost_enabled"):
        flag(io, sd, k)
    u32(io, sd, "recharge_boost_per_second")
    u32(io, sd, "recharge_boost_delay")
    byte(io, sd, "demo_mode")
    flag(io, sd, "enable_team_demos")
    u32(io, sd, "goal_base_threshold_y")
    flag(io, sd, "boost_pads_enabled")
    vec3(io, sd.gravity_bt)
    expect(io.count(NUM_DYN), NUM_DYN, "dynamic bodies")
    for d in range(NUM_DYN):
        u32(io, sd.dyn_body, d)
    vec3(io, sd.grid_min_pos)
    vec3(io, sd.grid_max_pos)
    u32(io, sd, "grid_cell_size")
    u32(io, sd, "grid_cell_size_sq")
    for k in range(3):
        u32(io, sd.grid_num_cells, k)
    vec3(io, sd.sap_world_aabb_min)
    vec3(io, sd.sap_quantize)
    for k in ("sap_handle_mask", "sap_sentinel", "sap_max_handles"):
        sd.set(k, io.u16v(sd.get(k) & 0xFFFF))
    u32(io, sd, "sap_world_half_extent")
    tag(io, b"BODY")
    expect(io.count(NUM_BODIES), NUM_BODIES, "bodies")
    mesh_tris = [0] * NUM_BODIES
    for i in range(NUM_BODIES):
        b = sd.bodies[i]
        u32(io, b, "world_array_idx")
        byte(io, b, "user_idx")
        u32(io, b, "user_pointer")
        u32(io, b, "broadphase_handle")
        byte(io, b, "filter_group")
        byte(io, b, "filter_mask")
        u32(io, b, "mass")
        u32(io, b, "inv_mass")
        vec3(io, b.inv_inertia_local)
        vec3(io, b.inv_mass_splat)
        for k in ("friction", "restitution", "contact_processing_threshold", "contact_breaking_threshold", "linear_damping",
                  "linear_sleeping_threshold", "angular_sleeping_threshold"):
            u32(io, b, k)
        aff3(io, b.pose)
        byte(io, b, "shape_kind")
        kind = b.shape_kind
        if kind == 0:
            u32(io, b, "mesh_tri_count")
            mesh_tris[i] = b.mesh_tri_count
        elif kind == 2:
            vec3(io, b.sphere_implicit_dim)
            u32(io, b, "sphere_margin")
        elif kind == 3:
            vec3(io, b.box_half_extents)
            u32(io, b, "box_margin")
            aff3(io, b.child_trans)
            aabb(io, b.compound_local_aabb)
        elif kind != 1:
            io.fail("unknown shape kind")
            raise DumpError(io.err)
    for d in range(NUM_DYN):
        bi = sd.dyn_body[d]
        if bi >= NUM_BODIES:
            io.fail("dynamic body index out of range")
            raise DumpError(io.err)
        sd.dyn_handle[d] = sd.bodies[bi].broadphase_handle
    tag(io, b"MESH")
    expect(io.count(NUM_MESHES), NUM_MESHES, "meshes")
    tf = nf = lf = 0
    for mi_ in range(NUM_MESHES):
        mi = sd.meshes[mi_]
        u32(io, mi, "body")
        aabb(io, mi.aabb_ident_cache)
        nt = io.count(mi.tri_count)
        t0 = tf if R else mi.tri_first
        if t0 + nt > MAX_TRIS:
            io.fail("triangles over the StaticData size")
            raise DumpError(io.err)
        mi.tri_first, mi.tri_count = t0, nt
        bulk(io, sd, "tris", TRI, t0, nt, "12I")
        aabb(io, mi.root_aabb)
        nn = io.count(mi.node_count)
        n0 = nf if R else mi.node_first
        if n0 + nn > MAX_NODES:
            io.fail("BVH nodes over the StaticData size")
            raise DumpError(io.err)
        mi.node_first, mi.node_count = n0, nn
        bulk(io, sd, "nodes", WIDE_NODE, n0, nn, "24I4IBI")
        nl = io.count(mi.leaf_count)
        l0 = lf if R else mi.leaf_first
        if l0 + nl > MAX_LEAVES:
            io.fail("BVH leaves over the StaticData size")
            raise DumpError(io.err)
        mi.leaf_first, mi.leaf_count = l0, nl
        bulk(io, sd, "leaves", LEAF, l0, nl, "7I")
        ni = io.count(nt)
        if ni != nt:
            io.fail("one triangle info per triangle expected")
            raise DumpError(io.err)
        bulk(io, sd, "infos", TRI_INFO, t0, ni, "B3I")
        tf, nf, lf = t0 + nt, n0 + nn, l0 + nl
    if R and (tf, nf, lf) != (MAX_TRIS, MAX_NODES, MAX_LEAVES):
        io.fail("mesh totals differ from StaticData sizes")
        raise DumpError(io.err)
    for k in range(NUM_MESHES):
        mi = sd.meshes[k]
        if mi.body >= NUM_BODIES or mi.tri_count != mesh_tris[mi.body]:
            io.fail("mesh triangle count differs from its body record")
            raise DumpError(io.err)
    tag(io, b"PLAN")
    expect(io.count(NUM_PLANES), NUM_PLANES, "planes")
    for k in range(NUM_PLANES):
        p = sd.planes[k]
        u32(io, p, "body")
        vec3(io, p.plane_normal)
        flag(io, p, "is_single_axis")
        u32(io, p, "single_axis_idx")
        flag(io, p, "single_axis_backwards")
        aabb(io, p.aabb_ident_cache)
        aabb(io, p.aabb_cache)
    tag(io, b"CELL")
    occupied = [c for c in range(NUM_GRID_CELLS) if sd.cells[c].count > 0] if not R else []
    m = io.count(len(occupied))
    first = 0
    for k in range(m):
        cell = io.u32v(0 if R else occupied[k])
        cnt = io.u32v(0 if R else sd.cells[cell].count)
        at = first if R else sd.cells[cell].first
        if cell >= NUM_GRID_CELLS or at + cnt > MAX_CELL_ENTRIES:
            io.fail("static ray cells over the StaticData size")
            raise DumpError(io.err)
        sd.cells[cell].first, sd.cells[cell].count = at, cnt
        for j in range(cnt):
            u32(io, sd.cell_handles, at + j)
        first = at + cnt
    if R and first != MAX_CELL_ENTRIES:
        io.fail("static ray-cell entries differ from StaticData size")
        raise DumpError(io.err)
    tag(io, b"CARS")
    expect(io.count(NUM_CARS), NUM_CARS, "cars")
    for c in range(NUM_CARS):
        cc = sd.cars[c]
        u32(io, cc, "car_idx")
        byte(io, cc, "team")
        u32(io, cc, "rigid_body_idx")
        flag(io, cc, "three_wheels")
        vec3(io, cc.hitbox_size)
        vec3(io, cc.hitbox_pos_offset)
        for w in range(NUM_WHEELS):
            wc = cc.wheels[w]
            vec3(io, wc.chassis_connection_point_cs)
            for k in ("suspension_rest_length_1", "wheels_radius", "suspension_force_scale", "real_ray_length"):
                u32(io, wc, k)
    tag(io, b"PADS")
    expect(io.count(NUM_PADS), NUM_PADS, "pads")
    u32(io, sd, "max_pad_z")
    for p in range(NUM_PADS):
        pc = sd.pads[p]
        vec3(io, pc.pos)
        flag(io, pc, "is_big")
        for k in ("box_radius", "cyl_radius", "max_cooldown", "boost_amount"):
            u32(io, pc, k)
        aabb(io, pc.aabb)
    tag(io, b"PROX")
    expect(io.count(NUM_HANDLES), NUM_HANDLES, "proxies")
    for h in range(NUM_HANDLES):
        p = sd.proxies[h]
        u32(io, p, "client_obj_idx")
        byte(io, p, "filter_group")
        byte(io, p, "filter_mask")
        u32(io, p, "unique_id")
        aabb(io, p.aabb)
        u32(io, p, "cell_idx")
        for k in range(3):
            u32(io, p.indices, k)
    if io.err is not None:
        raise DumpError(io.err)


def _expand(fmt: str):
    out, num = [], ""
    for ch in fmt:
        if ch.isdigit():
            num += ch
        else:
            out += [ch] * int(num or 1)
            num = ""
    return out


def bulk(io, sd, name, t, first, n, fields):
    """A run of n records of sd.<name> from index `first`, each in the dump as `fields` (struct codes, one per word of
    the record in memory order; B for a word written as one byte)."""
    base = sd.t.fields[name][0] + first * t.size
    codes = _expand(fields)
    words = t.size // 4
    assert len(codes) == words
    rec = struct.Struct("<" + "".join(codes))
    if io.READ:
        data = io.rawv(bytes(rec.size * n))
        for i in range(n):
            struct.pack_into(f"<{words}I", sd.b, base + i * t.size, *rec.unpack_from(data, i * rec.size))
    else:
        mem = np.frombuffer(bytes(sd.b[base:base + n * t.size]), np.uint32).reshape(n, words)
        byte_cols = [j for j, c in enumerate(codes) if c == "B"]
        for i in range(n):
            vals = [int(x) for x in mem[i]]
            for j in byte_cols:
                vals[j] &= 0xFF
            io.out += rec.pack(*vals)


def write_static(sd_words: np.ndarray):
    """(the static dump bytes, config_hash) of a StaticData, in the V3 side's export_static layout."""
    sd = V(bytearray(np.ascontiguousarray(sd_words, np.uint32).tobytes()), 0, STATIC_DATA)
    w = Wr()
    io_static(w, sd)
    payload = bytes(w.out)
    ranges = list(zip(w.marks, w.marks[1:] + [len(payload)]))
    cfg = b"".join(payload[a:b] for k, (a, b) in enumerate(ranges) if k in (0, 1, 3, 5, 6))
    counts = [NUM_BODIES, NUM_DYN, NUM_MESHES, sum(sd.meshes[m].tri_count for m in range(NUM_MESHES)),
              sum(sd.meshes[m].node_count for m in range(NUM_MESHES)), sum(sd.meshes[m].leaf_count for m in range(NUM_MESHES)),
              sum(sd.meshes[m].tri_count for m in range(NUM_MESHES)), NUM_PLANES, NUM_CARS, NUM_PADS, NUM_GRID_CELLS,
              sum(sd.cells[c].count for c in range(NUM_GRID_CELLS))]
    head = b"V3STATIC" + struct.pack("<IQQ12I", 3, fnv1a64(payload), len(payload), *counts)
    return head + payload, fnv1a64(cfg)


def parse_static(data: bytes) -> np.ndarray:
    """dump.rs:947-1012, except table_sin, which stays zero here (the importer fills it from its own sine)."""
    if len(data) < 76 or data[:8] != b"V3STATIC":
        raise DumpError("not a static dump (magic)")
    version = struct.unpack_from("<I", data, 8)[0]
    if version != 3:
        raise DumpError(f"unsupported static dump version {version} (need 3: re-vendor V3)")
    h, plen = struct.unpack_from("<QQ", data, 12)
    if plen != len(data) - 76:
        raise DumpError("static dump payload length mismatch")
    if fnv1a64(data[76:]) != h:
        raise DumpError("static dump payload hash mismatch")
    counts = struct.unpack_from("<12I", data, 28)
    want = (NUM_BODIES, NUM_DYN, NUM_MESHES, MAX_TRIS, MAX_NODES, MAX_LEAVES, MAX_TRIS, NUM_PLANES, NUM_CARS, NUM_PADS,
            NUM_GRID_CELLS, MAX_CELL_ENTRIES)
    for i, (got, w) in enumerate(zip(counts, want)):
        if got != w:
            raise DumpError(f"static dump count {i} is {got}; StaticData is sized for {w} (the project's 16 Soccar meshes)")
    sd = V(bytearray(STATIC_DATA.size), 0, STATIC_DATA)
    r = Rd(bytes(data[76:]))
    io_static(r, sd)
    if r.remaining():
        raise DumpError(f"{r.remaining()} trailing bytes in the static dump")
    return np.frombuffer(bytes(sd.b), np.uint32).copy()
