"""The FP64-free correctly rounded libm against the reference's correctly rounded libm (CORE-MATH ports in
cuda/common/libm_cr.cuh), on seeded samples and special values (CPU); all 2^32 inputs of sin, cos and tan are checked
on the GPU (test_gpu.py) against chunk hashes of the reference's values (tests/golden/libm_chunk_hashes.json)."""
import ctypes
import os

import numpy as np
import pytest

from conftest import PROBE_SO

SPECIAL = np.array([0.0, -0.0, 1e-45, -1e-45, 1.1754944e-38, 1e-10, 1e-5, 0.5, 1.0, -1.0, 2.0, 3.1415927, 1.5707964, 0.7853982,
                    100.0, 1e5, 1e10, 1e20, 3.4028235e38, -3.4028235e38, np.inf, -np.inf, np.nan, 7.0, 0.1, 1.0e-3], np.float32)


@pytest.fixture(scope="module")
def probe():
    if not os.path.exists(PROBE_SO):
        pytest.skip("oracle/_ref not built")
    L = ctypes.CDLL(PROBE_SO)
    for f in ("rsref_sinf", "rsref_cosf", "rsref_tanf"):
        getattr(L, f).restype = ctypes.c_float
        getattr(L, f).argtypes = [ctypes.c_float]
    for f in ("rsref_atan2f", "rsref_powf", "rsref_atan2_64_f", "rsref_hypot64_f"):
        getattr(L, f).restype = ctypes.c_float
        getattr(L, f).argtypes = [ctypes.c_float, ctypes.c_float]
    for f in ("rsref_atan2f_batch", "rsref_atan2_64_f_batch", "rsref_hypot64_f_batch"):
        getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_ulonglong]
    return L


def mine(rsx, fn, a, b=None):
    a = np.ascontiguousarray(a, np.float32)
    out = np.zeros_like(a)
    fp = ctypes.POINTER(ctypes.c_float)
    bb = np.ascontiguousarray(b, np.float32) if b is not None else a
    rc = rsx.lib().rsx_libm_host(fn, a.ctypes.data_as(fp), bb.ctypes.data_as(fp), out.ctypes.data_as(fp), a.size)
    assert rc == 0
    return out


def same(x, y):
    xb, yb = x.view(np.uint32), y.view(np.uint32)
    nan = (np.isnan(x) & np.isnan(y))
    return (xb == yb) | nan


@pytest.mark.parametrize("fn,name", [(0, "rsref_sinf"), (1, "rsref_cosf"), (2, "rsref_tanf")])
def test_unary_matches_reference(rsx, probe, fn, name):
    rng = np.random.default_rng(fn)
    x = np.concatenate([rng.integers(0, 2 ** 32, 40000, dtype=np.uint64).astype(np.uint32).view(np.float32),
                        rng.uniform(-10, 10, 20000).astype(np.float32), SPECIAL])
    want = np.array([getattr(probe, name)(float(v)) for v in x], np.float32)
    got = mine(rsx, fn, x)
    bad = ~same(want, got)
    assert not bad.any(), f"{bad.sum()} mismatches, first x={x[bad][:4]}"


@pytest.mark.parametrize("fn,name", [(3, "rsref_atan2f"), (4, "rsref_powf"), (5, "rsref_atan2_64_f"), (6, "rsref_hypot64_f")])
def test_binary_matches_reference(rsx, probe, fn, name):
    rng = np.random.default_rng(10 + fn)
    n = 30000
    a = np.concatenate([rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32).view(np.float32),
                        rng.uniform(-1, 1, n).astype(np.float32), np.repeat(SPECIAL, SPECIAL.size)])
    b = np.concatenate([rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32).view(np.float32),
                        rng.uniform(-1, 1, n).astype(np.float32), np.tile(SPECIAL, SPECIAL.size)])
    if fn == 4:  # pow: positive bases near 1 and small exponents as in the damping factor, plus the random pairs
        a[n:2 * n] = rng.uniform(0.0, 4.0, n).astype(np.float32)
        b[n:2 * n] = rng.uniform(-30, 30, n).astype(np.float32)
    f = getattr(probe, name)
    want = np.array([f(float(u), float(v)) for u, v in zip(a, b)], np.float32)
    got = mine(rsx, fn, a, b)
    bad = ~same(want, got)
    assert not bad.any(), f"{bad.sum()} mismatches, first a={a[bad][:3]} b={b[bad][:3]}"


@pytest.mark.parametrize("fn,name", [(3, "rsref_atan2f_batch"), (5, "rsref_atan2_64_f_batch"), (6, "rsref_hypot64_f_batch")])
def test_fast_path_domains(rsx, probe, fn, name):
    """2M pairs in the double-float fast paths' domains (atan2: operands in [2^-63, 2^64), exponents at most 60 apart;
    hypot: [2^-36, 2^61)): near the diagonal, near the axes, all quadrants, and the game's magnitudes; atan2f, the
    auto-flip's float(double atan2) and float(double hypot), bit for bit against the reference."""
    rng = np.random.default_rng(77)
    n = 400000
    sign = lambda k: np.where(rng.integers(0, 2, k) == 1, np.uint32(0x80000000), np.uint32(0))
    mant = lambda k: rng.integers(0, 1 << 23, k).astype(np.uint32)
    parts_y, parts_x = [], []
    e1 = rng.integers(107, 148, n)
    parts_y.append(e1)
    parts_x.append(rng.integers(107, 148, n))
    e2 = rng.integers(120, 130, n)  # near the diagonal
    parts_y.append(e2)
    parts_x.append(e2)
    e3 = rng.integers(127, 137, n)  # near the axes
    parts_y.append(e3)
    parts_x.append(e3 - rng.integers(0, 61, n))
    e4 = rng.integers(64, 191, n)
    parts_y.append(e4)
    parts_x.append(np.clip(e4 + rng.integers(-60, 61, n), 64, 190))
    ey = np.concatenate(parts_y).astype(np.uint32)
    ex = np.concatenate(parts_x).astype(np.uint32)
    m = ey.size
    my = mant(m)
    mx = mant(m)
    near = slice(n, 2 * n)
    mx[near] = (my[near] + rng.integers(-32, 33, n).astype(np.uint32)) & np.uint32(0x7FFFFF)
    y = (sign(m) | (ey << np.uint32(23)) | my).view(np.float32)
    x = (sign(m) | (ex << np.uint32(23)) | mx).view(np.float32)
    y = np.concatenate([y, rng.uniform(-3000, 3000, n).astype(np.float32)])
    x = np.concatenate([x, rng.uniform(-3000, 3000, n).astype(np.float32)])
    want = np.zeros_like(y)
    getattr(probe, name)(y.ctypes.data, x.ctypes.data, want.ctypes.data, y.size)
    got = mine(rsx, fn, y, x)
    bad = ~same(want, got)
    assert not bad.any(), f"{bad.sum()} mismatches, first y={y[bad][:3]} x={x[bad][:3]}"


def test_damping_factor_exact(rsx, probe):
    # the one pow the physics calls: (1 - linear_damping)^(1/120)
    for damping in (0.03, 0.0305, 0.1, 0.5):
        x = np.float32(1.0) - np.float32(damping)
        y = np.float32(1.0) / np.float32(120.0)
        assert probe.rsref_powf(float(x), float(y)) == mine(rsx, 4, np.array([x]), np.array([y]))[0]


def test_host_hash_matches_reference_chunk(rsx):
    import json

    path = os.path.join(os.path.dirname(__file__), "golden", "libm_chunk_hashes.json")
    if not os.path.exists(path):
        pytest.skip("libm chunk hashes not generated")
    with open(path) as f:
        gold = json.load(f)
    L = rsx.lib()
    L.rsx_libm_hash_host.restype = ctypes.c_uint64
    L.rsx_libm_hash_host.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32]
    for fn, name in enumerate(("sin", "cos", "tan")):
        # chunks 0x3F (inputs around 0.5..2) and 0xC0 (negative, moderate) recomputed on the host
        for chunk in (0x3F, 0xC0):
            assert "%016x" % L.rsx_libm_hash_host(fn, chunk << 24, 1 << 24) == gold[name][chunk]
