"""Shared test setup: the `gpu` marker, the package path, and the oracle.

The oracle is the reference's own correctly rounded CPU simulator (crates/rocketsim-cuda/csrc/phase.cpp over the
reference's cuda/ headers), built from its sources by oracle/Makefile into oracle/_ref/.  Tests use it to check
against only; when it is absent (a machine that never had the reference sources), the committed golden fixtures of
tests/golden/ stand in for it.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "rocketsim-cuda_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, os.path.join(ROOT, "tests"))
ORACLE_SO = os.path.join(ROOT, "oracle", "_ref", "librsref.so")
PROBE_SO = os.path.join(ROOT, "oracle", "_ref", "librsprobe.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


class Oracle:
    """ctypes view of the reference's CPU build (test infrastructure; never on a product path)."""

    def __init__(self, path=ORACLE_SO):
        self.L = ctypes.CDLL(path)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        self.L.rscuda_phase.argtypes = [ctypes.c_int, u32p, u32p]
        self.L.rscuda_step_tick.argtypes = [u32p, u32p]
        self.L.rscuda_step_ticks.argtypes = [u32p, u32p, u32p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32), u32p]
        for f in ("lf_arena_words", "lf_tick_words", "lf_static_words"):
            getattr(self.L, f).restype = ctypes.c_uint64
        self.L.lf_aosoa_index.restype = ctypes.c_uint64
        self.L.lf_aosoa_index.argtypes = [ctypes.c_uint32, ctypes.c_int]
        self.L.lf_aosoa_words.restype = ctypes.c_uint64
        self.L.lf_aosoa_words.argtypes = [ctypes.c_uint32]

    @staticmethod
    def p(a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))

    def phase(self, k, state, sd):
        return self.L.rscuda_phase(k, self.p(state), self.p(sd))

    def decide(self, state, sd, controls16, ticks=8):
        """One decision in place (rscuda_step_ticks); returns the scored tick."""
        sc = ctypes.c_uint32(0)
        self.L.rscuda_step_ticks(self.p(state), self.p(sd), self.p(np.ascontiguousarray(controls16)), ticks, ctypes.byref(sc), None)
        return sc.value

    def run(self, states, sd, controls):
        """Decisions of many arenas in place: states (n, 2784), controls (n, 16); returns scored ticks."""
        out = np.zeros(states.shape[0], np.uint32)
        for a in range(states.shape[0]):
            out[a] = self.decide(states[a], sd, controls[a])
        return out


@pytest.fixture(scope="session")
def oracle():
    if not os.path.exists(ORACLE_SO):
        pytest.skip("oracle/_ref not built (no reference sources on this machine): golden fixtures cover it")
    return Oracle()


@pytest.fixture(scope="session")
def rsx():
    import rsx as m

    m.lib()
    return m


@pytest.fixture(scope="session")
def world(rsx):
    return rsx.build_static(7, 0, 0)
