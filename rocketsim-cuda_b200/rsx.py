"""Python host side of the soccar decision step: a ctypes mirror of the reference's Rust host crate API
(crates/rocketsim-cuda/src/device.rs SimDevice: new, upload_static, upload_states, alloc_states, download_states,
upload_controls, sim8, step_tick, phase, identity) over the C ABI of librsx.so (include/rsx.h).

Device memory for controls / results comes from torch (plumbing only); states and static data are owned by the
library's handles.  Nothing here computes physics: every step runs the CUDA kernels, and a missing library is an error.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librsx.so")

ARENA_WORDS = 2784
TICK_WORDS = 2567
STATIC_WORDS = 317895
TICKS_PER_DECISION = 8
SCORED_MASK = 0xFF
UNIMPLEMENTED = 0x80000000
OVERFLOW = 0x40000000
SIM8_BLOCK = 32
MAX_BLOCK = 64
NUM_CARS = 2
CONTROL_WORDS = 8

# offsets of a few words of ArenaState (the reference's layout)
W_EVENTS = TICK_WORDS - 1
MIX_HEADLINE = (0.20, 0.50, 0.15, 0.10, 0.05)  # kickoff, open play, head-on, pinch, pad contention
MIX_KICKOFF = (1.0, 0.0, 0.0, 0.0, 0.0)
MIX_CONTACT_HEAVY = (0.10, 0.20, 0.30, 0.40, 0.0)

_lib = None


class RsxError(RuntimeError):
    pass


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RsxError(f"librsx.so is not built ({LIB_PATH}); run `make -C rocketsim-cuda_b200`")
        L = ctypes.CDLL(LIB_PATH)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.rsx_arena_words.restype = ctypes.c_uint64
        L.rsx_tick_words.restype = ctypes.c_uint64
        L.rsx_static_words.restype = ctypes.c_uint64
        L.rsx_aosoa_words.restype = ctypes.c_uint64
        L.rsx_aosoa_words.argtypes = [ctypes.c_uint32]
        L.rsx_aosoa_index.restype = ctypes.c_uint64
        L.rsx_aosoa_index.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.rsx_aosoa_pack.argtypes = [u32p, ctypes.c_uint32, u32p]
        L.rsx_aosoa_unpack.argtypes = [u32p, ctypes.c_uint32, u32p]
        L.rsx_last_error.restype = ctypes.c_char_p
        L.rsx_build_static.argtypes = [u32p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        L.rsx_make_states.argtypes = [u32p, u32p, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_float)]
        L.rsx_make_states_multi.argtypes = [u32p, ctypes.c_uint32, ctypes.c_void_p, u32p, ctypes.c_uint32, ctypes.c_uint64,
                                            ctypes.POINTER(ctypes.c_float)]
        fp = ctypes.POINTER(ctypes.c_float)
        L.rsx_libm_host.argtypes = [ctypes.c_int, fp, fp, fp, ctypes.c_uint64]
        L.rsx_libm_hash_host.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32]
        L.rsx_libm_hash_host.restype = ctypes.c_uint64
        L.rsx_libm_chunk_hashes.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
        L.rsx_host_phase.argtypes = [ctypes.c_int, u32p, u32p]
        L.rsx_host_decide.argtypes = [u32p, u32p, u32p]
        L.rsx_host_decide.restype = ctypes.c_uint32
        vp = ctypes.c_void_p
        L.rsx_device_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
        L.rsx_device_destroy.argtypes = [vp]
        L.rsx_sync.argtypes = [vp]
        L.rsx_device_stream.argtypes = [vp]
        L.rsx_device_stream.restype = vp
        L.rsx_static_upload.argtypes = [vp, u32p, ctypes.c_uint32, ctypes.POINTER(vp)]
        L.rsx_static_free.argtypes = [vp]
        L.rsx_static_device_ptr.argtypes = [vp]
        L.rsx_static_device_ptr.restype = vp
        L.rsx_states_alloc.argtypes = [vp, ctypes.c_uint32, ctypes.POINTER(vp)]
        L.rsx_states_free.argtypes = [vp]
        L.rsx_states_upload.argtypes = [vp, vp, u32p]
        L.rsx_states_download.argtypes = [vp, vp, u32p]
        L.rsx_states_device_ptr.argtypes = [vp]
        L.rsx_states_device_ptr.restype = vp
        L.rsx_sim8.argtypes = [vp, vp, vp, vp, vp, ctypes.c_uint32, vp]
        L.rsx_sim8_raw.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, ctypes.c_uint32, vp, vp]
        L.rsx_step_tick.argtypes = [vp, vp, vp, vp]
        L.rsx_phase.argtypes = [vp, ctypes.c_int, vp, vp, vp]
        L.rsx_identity.argtypes = [vp, vp, vp, ctypes.c_uint32, ctypes.c_int]
        L.rsx_sim8_multi_raw.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, vp, ctypes.c_uint32, vp]
        L.rsx_sim8_persistent_raw.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32,
                                              ctypes.c_uint32, vp]
        L.rsx_sim8_persistent_ex.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32,
                                             ctypes.c_uint32, ctypes.c_uint32, vp, vp]
        L.rsx_sim8_lockstep_raw.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32,
                                            ctypes.c_uint32, vp]
        L.rsx_sim8_lockstep_ex.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.c_uint32, ctypes.c_uint32, vp]
        L.rsx_copy_raw.argtypes = [vp, vp, ctypes.c_uint64, vp]
        L.rsx_make_states_at.argtypes = [u32p, ctypes.c_uint32, vp, vp, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_float), u32p]
        L.rsx_l2_persist_raw.argtypes = [vp, ctypes.c_uint64, ctypes.c_float, vp]
        L.rsx_reset_arenas_raw.argtypes = [vp, ctypes.c_uint32, vp, vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_float), vp, vp, vp, vp]
        L.rsx_pad_mirror.argtypes = [u32p, ctypes.c_uint32, vp]
        L.rsx_observe_raw.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_float), vp, vp, vp]
        szp = ctypes.POINTER(ctypes.c_size_t)
        tp = ctypes.POINTER(V3Template)
        L.rsx_v3_fnv1a64.argtypes = [vp, ctypes.c_size_t]
        L.rsx_v3_fnv1a64.restype = ctypes.c_uint64
        L.rsx_v3_parse_static.argtypes = [vp, ctypes.c_size_t, u32p]
        L.rsx_v3_write_static.argtypes = [u32p, vp, ctypes.c_size_t, szp]
        L.rsx_v3_config_hash.argtypes = [u32p, ctypes.POINTER(ctypes.c_uint64)]
        L.rsx_v3_template_init.argtypes = [u32p, tp]
        L.rsx_v3_parse_arena.argtypes = [vp, ctypes.c_size_t, u32p, u32p, tp]
        L.rsx_v3_write_arena.argtypes = [u32p, u32p, tp, vp, ctypes.c_size_t, szp]
        _lib = L
    return _lib


class V3Template(ctypes.Structure):
    """What an ArenaState leaves out of a V3 arena dump (rsx_v3_template; the reference's dump.rs Template)."""
    _fields_ = [("config_hash", ctypes.c_uint64), ("static_body", (ctypes.c_uint8 * 219) * 23), ("num_handles", ctypes.c_uint16),
                ("next_new_handle", ctypes.c_uint16), ("manifold_stride", ctypes.c_uint32), ("ball_other", ctypes.c_uint8 * 24),
                ("ball_other_set", ctypes.c_uint32)]


def _p(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def check(rc: int, what: str) -> None:
    if rc < 0:
        raise RsxError(f"{what} failed ({rc}): {lib().rsx_last_error().decode(errors='replace')}")


# ---- host-side data ----------------------------------------------------------------------------------------------
def build_static(seed: int = 7, preset0: int = 0, preset1: int = 0) -> np.ndarray:
    """One StaticData of the synthetic soccar world for the car pairing (preset0, preset1)."""
    sd = np.zeros(STATIC_WORDS, np.uint32)
    check(lib().rsx_build_static(_p(sd), seed, preset0, preset1), "rsx_build_static")
    return sd


def make_states(sd: np.ndarray, n: int, seed: int, mix: Sequence[float] = MIX_HEADLINE) -> np.ndarray:
    """n seeded start states (n x 2784 words)."""
    st = np.zeros((n, ARENA_WORDS), np.uint32)
    m = (ctypes.c_float * 5)(*mix)
    check(lib().rsx_make_states(_p(sd), _p(st), n, seed, m), "rsx_make_states")
    return st


def make_states_multi(sds: np.ndarray, sd_index: np.ndarray, seed: int, mix: Sequence[float] = MIX_HEADLINE) -> np.ndarray:
    """Start states with a car pairing per arena: sds (count, 317895), sd_index (n,) uint8."""
    sds = np.ascontiguousarray(sds.reshape(-1, STATIC_WORDS), np.uint32)
    idx = np.ascontiguousarray(sd_index, np.uint8)
    n = idx.shape[0]
    st = np.zeros((n, ARENA_WORDS), np.uint32)
    m = (ctypes.c_float * 5)(*mix)
    check(lib().rsx_make_states_multi(_p(sds.reshape(-1)), sds.shape[0], idx.ctypes.data_as(ctypes.c_void_p), _p(st), n, seed, m),
          "rsx_make_states_multi")
    return st


def make_states_at(sds: np.ndarray, sd_index: np.ndarray, arena_index: np.ndarray, seed: int, mix: Sequence[float]) -> np.ndarray:
    """The start states of the arenas `arena_index` (their car pairings `sd_index`): the words make_states_multi and the
    device reset give those arenas."""
    sds = np.ascontiguousarray(sds.reshape(-1, STATIC_WORDS), dtype=np.uint32)
    si = np.ascontiguousarray(sd_index, dtype=np.uint8)
    ai = np.ascontiguousarray(arena_index, dtype=np.uint32)
    out = np.zeros((ai.size, ARENA_WORDS), np.uint32)
    m = (ctypes.c_float * 5)(*mix)
    check(lib().rsx_make_states_at(_p(sds.reshape(-1)), sds.shape[0], si.ctypes.data_as(ctypes.c_void_p), ai.ctypes.data_as(ctypes.c_void_p),
                                   ai.size, seed, m, _p(out)), "rsx_make_states_at")
    return out


OBS_DIM = 104
REWARD_TERMS = 8


def pad_mirror(sds: np.ndarray) -> np.ndarray:
    """For each StaticData, the pad at the mirror image (-x, -y, z) of each pad (count x 34 u8): car 1's pad order in
    its observation."""
    sds = np.ascontiguousarray(sds.reshape(-1, STATIC_WORDS), np.uint32)
    out = np.zeros((sds.shape[0], 34), np.uint8)
    check(lib().rsx_pad_mirror(_p(sds.reshape(-1)), sds.shape[0], out.ctypes.data_as(ctypes.c_void_p)), "rsx_pad_mirror")
    return out


# ---- V3 dumps (the reference's crates/rocketsim-cuda/src/dump.rs) ------------------------------------------------
E_FORMAT = -5


def _bytes_arg(b: bytes):
    buf = ctypes.create_string_buffer(bytes(b), len(b))
    return buf, len(b)


def _write_out(fn, *args) -> bytes:
    n = ctypes.c_size_t(0)
    fn(*args, None, 0, ctypes.byref(n))  # asks for the size
    out = ctypes.create_string_buffer(n.value)
    check(fn(*args, out, n.value, ctypes.byref(n)), fn.__name__)
    return out.raw[:n.value]


def v3_fnv1a64(b: bytes) -> int:
    buf, n = _bytes_arg(b)
    return int(lib().rsx_v3_fnv1a64(buf, n))


def v3_parse_static(b: bytes) -> np.ndarray:
    """A V3STATIC (version 3) dump as StaticData words (parse_static)."""
    buf, n = _bytes_arg(b)
    sd = np.zeros(STATIC_WORDS, np.uint32)
    check(lib().rsx_v3_parse_static(buf, n, _p(sd)), "rsx_v3_parse_static")
    return sd


def v3_write_static(sd: np.ndarray) -> bytes:
    sd = np.ascontiguousarray(sd, np.uint32)
    return _write_out(lib().rsx_v3_write_static, _p(sd))


def v3_config_hash(sd: np.ndarray) -> int:
    sd = np.ascontiguousarray(sd, np.uint32)
    h = ctypes.c_uint64(0)
    check(lib().rsx_v3_config_hash(_p(sd), ctypes.byref(h)), "rsx_v3_config_hash")
    return int(h.value)


def v3_template(sd: np.ndarray) -> V3Template:
    """A template for a StaticData without a V3 dump (the synthetic world)."""
    sd = np.ascontiguousarray(sd, np.uint32)
    t = V3Template()
    check(lib().rsx_v3_template_init(_p(sd), ctypes.byref(t)), "rsx_v3_template_init")
    return t


def v3_parse_arena(b: bytes, sd: np.ndarray):
    """A V3ARENA (version 2) dump as 2784 state words, and its template (parse_arena)."""
    sd = np.ascontiguousarray(sd, np.uint32)
    buf, n = _bytes_arg(b)
    st = np.zeros(ARENA_WORDS, np.uint32)
    t = V3Template()
    check(lib().rsx_v3_parse_arena(buf, n, _p(sd), _p(st), ctypes.byref(t)), "rsx_v3_parse_arena")
    return st, t


def v3_write_arena(state: np.ndarray, sd: np.ndarray, t: V3Template) -> bytes:
    """An ArenaState as a V3 arena dump (write_arena)."""
    state = np.ascontiguousarray(state, np.uint32)
    sd = np.ascontiguousarray(sd, np.uint32)
    return _write_out(lib().rsx_v3_write_arena, _p(state), _p(sd), ctypes.byref(t))


def aosoa_words(n: int) -> int:
    return int(lib().rsx_aosoa_words(n))


def pack(states: np.ndarray) -> np.ndarray:
    """n x 2784 ArenaStates -> AoSoA-32 words (numpy, vectorised: the layout of aosoa.cuh:17)."""
    n = states.shape[0]
    blocks = (n + 31) // 32
    pad = np.zeros((blocks * 32, ARENA_WORDS), np.uint32)
    pad[:n] = states
    return np.ascontiguousarray(pad.reshape(blocks, 32, ARENA_WORDS).transpose(0, 2, 1)).reshape(-1)


def unpack(words: np.ndarray, n: int) -> np.ndarray:
    blocks = (n + 31) // 32
    return np.ascontiguousarray(words.reshape(blocks, ARENA_WORDS, 32).transpose(0, 2, 1)).reshape(blocks * 32, ARENA_WORDS)[:n]


def _mix64(z: np.ndarray) -> np.ndarray:
    """SplitMix64's finaliser on uint64 arrays (wrapping)."""
    z = z + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def decision_controls(seed: int, decision: int, n: int) -> np.ndarray:
    """Deterministic controls of one decision for n arenas (the scheme of the reference's test controls,
    tests/common/mod.rs:27-44: a SplitMix hash per (decision, arena, car); axes in {-1, 0, 1} from 4-bit fields, jump /
    boost / handbrake from single bits).  Returns words (n, 16)."""
    with np.errstate(over="ignore"):
        a = np.arange(n, dtype=np.uint64)
        out = np.zeros((n, NUM_CARS, CONTROL_WORDS), np.uint32)
        for car in range(NUM_CARS):
            key = (np.uint64(seed) << np.uint64(48)) ^ (np.uint64(decision) << np.uint64(24)) ^ (a << np.uint64(1)) ^ np.uint64(car)
            h = _mix64(key)
            for k in range(5):
                out[:, car, k] = (((h >> np.uint64(4 * k)) % np.uint64(3)).astype(np.int64) - 1).astype(np.float32).view(np.uint32)
            for k in range(3):
                out[:, car, 5 + k] = ((h >> np.uint64(24 + k)) & np.uint64(1)).astype(np.uint32)
    return out.reshape(n, NUM_CARS * CONTROL_WORDS)


def random_controls(rng: np.random.Generator, n: int) -> np.ndarray:
    """Controls[n][2] as words: each axis uniform in {-1, 0, 1}, jump / boost / handbrake Bernoulli(0.5)."""
    c = np.zeros((n, NUM_CARS, CONTROL_WORDS), np.uint32)
    axes = rng.integers(-1, 2, size=(n, NUM_CARS, 5)).astype(np.float32)
    c[:, :, :5] = axes.view(np.uint32)
    c[:, :, 5:] = rng.integers(0, 2, size=(n, NUM_CARS, 3)).astype(np.uint32)
    return c.reshape(n, NUM_CARS * CONTROL_WORDS)


# ---- the device handle (SimDevice) --------------------------------------------------------------------------------
class SimDevice:
    def __init__(self, ordinal: int = 0):
        import torch  # device memory for controls and results

        self.torch = torch
        h = ctypes.c_void_p()
        check(lib().rsx_device_create(ordinal, ctypes.byref(h)), "rsx_device_create")
        self.h = h
        self.ordinal = ordinal
        self.device = torch.device("cuda", ordinal)

    def close(self):
        if self.h:
            lib().rsx_device_destroy(self.h)
            self.h = None

    def stream_ptr(self) -> int:
        return lib().rsx_device_stream(self.h)

    def upload_static(self, sds: np.ndarray) -> "DeviceStatic":
        sds = np.ascontiguousarray(sds.reshape(-1, STATIC_WORDS), dtype=np.uint32)
        h = ctypes.c_void_p()
        check(lib().rsx_static_upload(self.h, _p(sds.reshape(-1)), sds.shape[0], ctypes.byref(h)), "rsx_static_upload")
        return DeviceStatic(h, sds.shape[0])

    def alloc_states(self, n: int) -> "DeviceStates":
        h = ctypes.c_void_p()
        check(lib().rsx_states_alloc(self.h, n, ctypes.byref(h)), "rsx_states_alloc")
        return DeviceStates(h, n)

    def upload_states(self, states: np.ndarray) -> "DeviceStates":
        d = self.alloc_states(states.shape[0])
        words = pack(states)
        check(lib().rsx_states_upload(self.h, d.h, _p(words)), "rsx_states_upload")
        return d

    def download_words(self, d: "DeviceStates") -> np.ndarray:
        out = np.zeros(aosoa_words(d.n), np.uint32)
        check(lib().rsx_states_download(self.h, d.h, _p(out)), "rsx_states_download")
        return out

    def download_states(self, d: "DeviceStates") -> np.ndarray:
        return unpack(self.download_words(d), d.n)

    def upload_controls(self, controls: np.ndarray):
        """Controls as device words; the copy completes before this returns (the handle's launches follow it)."""
        t = self.torch.from_numpy(np.ascontiguousarray(controls.view(np.int32))).to(self.device)
        self.torch.cuda.current_stream(self.device).synchronize()
        return t

    def alloc_result(self, n: int):
        t = self.torch.zeros(n, dtype=self.torch.int32, device=self.device)
        self.torch.cuda.current_stream(self.device).synchronize()
        return t

    def sim8(self, states: "DeviceStates", sd: "DeviceStatic", controls, result, block: int = SIM8_BLOCK, trace=None) -> None:
        if not (1 <= block <= MAX_BLOCK):
            raise ValueError(f"sim8: block of {block} threads")
        if controls.numel() < states.n * 16 or result.numel() < states.n:
            raise ValueError("sim8: buffers too short")
        tp = trace.data_ptr() if trace is not None else None
        check(lib().rsx_sim8(self.h, states.h, sd.h, controls.data_ptr(), result.data_ptr(), block, tp), "rsx_sim8")

    def step_tick(self, states: "DeviceStates", sd: "DeviceStatic") -> np.ndarray:
        status = self.torch.zeros(states.n, dtype=self.torch.int32, device=self.device)
        check(lib().rsx_step_tick(self.h, states.h, sd.h, status.data_ptr()), "rsx_step_tick")
        self.sync()
        return status.cpu().numpy()

    def phase(self, k: int, states: "DeviceStates", sd: "DeviceStatic") -> np.ndarray:
        status = self.torch.zeros(states.n, dtype=self.torch.int32, device=self.device)
        check(lib().rsx_phase(self.h, k, states.h, sd.h, status.data_ptr()), "rsx_phase")
        self.sync()
        return status.cpu().numpy()

    def sync(self) -> None:
        check(lib().rsx_sync(self.h), "rsx_sync")


class DeviceStatic:
    def __init__(self, h, count):
        self.h = h
        self.count = count

    def ptr(self) -> int:
        return lib().rsx_static_device_ptr(self.h)

    def free(self):
        if self.h:
            lib().rsx_static_free(self.h)
            self.h = None


class DeviceStates:
    def __init__(self, h, n):
        self.h = h
        self.n = n

    def ptr(self) -> int:
        return lib().rsx_states_device_ptr(self.h)

    def free(self):
        if self.h:
            lib().rsx_states_free(self.h)
            self.h = None
