"""The reference's own GPU decision kernel, `sim8` (cuda/sim/sim.cu:95-104), for comparison runs only.

Test and measurement infrastructure, like the rest of oracle/: nothing on the product path imports this.  oracle/Makefile
(`make gpu`) compiles the reference's cuda/sim/sim.cu unchanged for sm_100a into oracle/_ref/sim8_ref.cubin with the
flags of the reference's build crate; this module loads that cubin through the CUDA driver API (ctypes on libcuda, in
the primary context torch uses) and launches `sim8(states, sd, controls, result, n)` the way the reference's host crate
does (crates/rocketsim-cuda/src/device.rs:155-171: one thread per arena, SIM8_BLOCK = 32 threads per block, grid
ceil(n / block)), after giving the context the reference's 8 KiB per-thread stack (crates/rocketsim-cuda/src/cuda.rs:
12-25).  The arena and static layouts are the same words as this project's, so the same device buffers serve both.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
CUBIN = os.path.join(HERE, "_ref", "sim8_ref.cubin")
SIM8_BLOCK = 32
STACK_BYTES = 8192
CU_LIMIT_STACK_SIZE = 0


def available() -> bool:
    return os.path.exists(CUBIN)


class RefSim8:
    """sim8 of the reference, loaded into the current device's primary context (torch must have initialised it)."""

    def __init__(self, device_index: int = 0):
        import torch

        torch.cuda.set_device(device_index)
        torch.cuda.init()
        torch.zeros(1, device=f"cuda:{device_index}")  # the primary context exists and is current on this thread
        self.cu = ctypes.CDLL("libcuda.so.1")
        ctx = ctypes.c_void_p()
        self._ck(self.cu.cuCtxGetCurrent(ctypes.byref(ctx)), "cuCtxGetCurrent")
        if not ctx.value:
            raise RuntimeError("no current CUDA context")
        self._ck(self.cu.cuCtxSetLimit(CU_LIMIT_STACK_SIZE, ctypes.c_size_t(STACK_BYTES)), "cuCtxSetLimit")
        self.mod = ctypes.c_void_p()
        self._ck(self.cu.cuModuleLoad(ctypes.byref(self.mod), CUBIN.encode()), "cuModuleLoad")
        self.fn = ctypes.c_void_p()
        self._ck(self.cu.cuModuleGetFunction(ctypes.byref(self.fn), self.mod, b"sim8"), "cuModuleGetFunction(sim8)")

    def _ck(self, rc, what):
        if rc != 0:
            name = ctypes.c_char_p()
            self.cu.cuGetErrorName(rc, ctypes.byref(name))
            raise RuntimeError(f"{what}: CUDA driver error {rc} ({name.value})")

    def sim8(self, d_states: int, n: int, d_static: int, d_controls: int, d_result: int, stream: int = 0, block: int = SIM8_BLOCK):
        """One decision of the n arenas of the AoSoA-32 buffer at d_states in place (reference sim8), async on `stream`."""
        if not 1 <= block <= 64:
            raise ValueError("sim8: block of 1..64 threads (SIM_MAX_BLOCK)")
        if n == 0:
            return
        args = [ctypes.c_void_p(d_states), ctypes.c_void_p(d_static), ctypes.c_void_p(d_controls), ctypes.c_void_p(d_result),
                ctypes.c_uint32(n)]
        params = (ctypes.c_void_p * len(args))(*[ctypes.cast(ctypes.pointer(a), ctypes.c_void_p) for a in args])
        grid = (n + block - 1) // block
        self._ck(self.cu.cuLaunchKernel(self.fn, grid, 1, 1, block, 1, 1, 0, ctypes.c_void_p(stream), params, None), "cuLaunchKernel(sim8)")

    def close(self):
        if self.mod:
            self.cu.cuModuleUnload(self.mod)
            self.mod = ctypes.c_void_p()
