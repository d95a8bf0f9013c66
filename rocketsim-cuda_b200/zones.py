"""Zone-timer profile of one decision of the headline workload (warp cycles per phase and per barrier, and with the
`all` library the simulator's inner markers), from librsx_zones.so / librsx_zones_all.so (`make -C rocketsim-cuda_b200
zones`).  Profiling only.

  python rocketsim-cuda_b200/zones.py [--all] [--arenas 65536] [--mix headline|contact] [--decisions 3]
"""
import argparse
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

NAMES = {0: "P1 car pre-tick head", 1: "P1 wheel rays", 2: "P1 wheel response", 3: "P1 car pre-tick tail", 10: "P3b pair heads",
         11: "P3b box-triangle SAT", 12: "P3b box BVH step", 13: "P3b box job tail", 14: "P3b sphere BVH step",
         15: "P3b sphere-triangle", 16: "P3b sphere job tail", 17: "  head: convex-plane", 18: "  head: sphere-box",
         19: "  head: box-box", 21: "  head: sphere job begin", 22: "  head: box job begin", 23: "  head: near tail",
         24: "  ray: box", 25: "  ray: sphere", 26: "  ray: plane", 27: "  ray: mesh", 28: "  ray: body setup",
         60: "copy-in (load_tick)", 61: "copy-out (store_tick)"}
for k, nm in enumerate(["P0", "P1", "P2", "P3a", "P3b", "P4", "P5", "P6", "P7", "P8"]):
    NAMES[40 + k] = "phase " + nm
    NAMES[50 + k] = "barrier after " + nm


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--all", action="store_true")
    ap.add_argument("--arenas", type=int, default=65536)
    ap.add_argument("--mix", default="headline", choices=["headline", "contact"])
    ap.add_argument("--decisions", type=int, default=3)
    args = ap.parse_args()
    import torch
    import rsx
    import bench

    Z = ctypes.CDLL(os.path.join(HERE, "librsx_zones_all.so" if args.all else "librsx_zones.so"))
    vp = ctypes.c_void_p
    Z.rsx_zones_decision.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, vp, vp]
    dev = rsx.SimDevice(0)
    n = args.arenas
    sds, idx, st = bench.world(rsx, n, 0, 1)
    if args.mix == "contact":
        st = rsx.make_states_multi(sds, idx, 1, rsx.MIX_CONTACT_HEAVY)
    dsd = dev.upload_static(sds)
    ds = dev.upload_states(st)
    didx = torch.from_numpy(idx).to(dev.device)
    res = torch.zeros(n, dtype=torch.int32, device=dev.device)
    counter = torch.zeros(1, dtype=torch.int32, device=dev.device)
    tot = np.zeros(64, np.float64)
    for d in range(args.decisions):
        ctl = dev.upload_controls(rsx.decision_controls(1000, d, n))
        out = np.zeros(64, np.uint64)
        rc = Z.rsx_zones_decision(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), res.data_ptr(), counter.data_ptr(), out.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"zone run failed ({rc})")
        tot += out.astype(np.float64)
    phases = sum(tot[40 + k] for k in range(10))
    barriers = sum(tot[50 + k] for k in range(10))
    print(f"{args.mix}, {n} arenas, {args.decisions} decisions: warp Gcycles in phases {phases / 1e9:.2f}, at barriers {barriers / 1e9:.2f}")
    for i in sorted(NAMES):
        if tot[i] > 0:
            print(f"  {NAMES[i]:28s} {tot[i] / 1e9:9.3f} G  {100 * tot[i] / phases:6.2f}% of phase cycles")


if __name__ == "__main__":
    main()
