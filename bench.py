#!/usr/bin/env python
"""Benchmark of the soccar 1v1 8-tick decision step on B200.

Metric: arena-ticks/s of one 8-tick decision over 65,536 arenas per GPU (the headline configuration: mixed start
states 20% kickoff / 50% open play / 15% head-on / 10% pinch / 5% pad contention, car pairings uniform over the 7 x 7
hitbox presets, random controls held for 8 ticks), bit-exact with the reference's CPU build.  A step is one decision of
every arena.  Seeded synthetic states over a seeded synthetic arena stand in for the reference's V3-played states and
the game's meshes (neither exists here).

  python bench.py [--gpus N --steps K --warmup W]          this implementation (one JSON line)
  python bench.py --impl reference ...                     the reference's own CPU build on the host's cores

`value` is device time of the decision kernels with states resident in HBM (max over ranks); `e2e` times the public
entry point with the controls copied from pinned host memory and the result words read back every step.  N > 1: one
process per GPU, each with its own 65,536 arenas (weak scaling); arenas are independent, so no collective touches the
data path (the timing max is the only reduction).
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rocketsim-cuda_b200"))

ARENAS = 65536
TICK_BYTES = 2567 * 4
ALG_BYTES_PER_ARENA_TICK = (TICK_BYTES * 2 + 64 + 4) / 8.0  # state in + out, controls, result, per tick
METRIC = "arena-ticks/s, 8-tick decision, 65,536 arenas: binned vs plain, bit-exact"
PRESETS = [(p, q) for p in range(7) for q in range(7)]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--arenas", type=int, default=ARENAS)
    ap.add_argument("--mode", default="plain", choices=["plain", "persistent"])
    ap.add_argument("--block", type=int, default=32)
    ap.add_argument("--cpu-sample", type=int, default=8192, help="arenas of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--seed", type=int, default=1)
    return ap.parse_args()


def world(rsx, n, rank, seed):
    """The 49 car pairings' StaticData, a pairing per arena, and the mixed start states."""
    sds = np.stack([rsx.build_static(7, p, q) for p, q in PRESETS])
    with np.errstate(over="ignore"):
        h = rsx._mix64(np.arange(n, dtype=np.uint64) + np.uint64((rank + 1) << 40))
    idx = (h % np.uint64(len(PRESETS))).astype(np.uint8)
    st = rsx.make_states_multi(sds, idx, seed + rank, rsx.MIX_HEADLINE)
    return sds, idx, st


def oracle_batch():
    path = os.path.join(ROOT, "oracle", "_ref", "librsbatch.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    L.rsref_run_batch.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                  ctypes.c_int, ctypes.c_void_p]
    return L


def cpu_run(L, rsx, sds, idx, st, decisions, seed):
    """The reference's CPU build over `st` (in place) for `decisions` decisions on all host threads; returns
    (arena-ticks/s, threads, seconds)."""
    n = st.shape[0]
    ctl = np.ascontiguousarray(np.stack([rsx.decision_controls(seed, d, n) for d in range(decisions)]))
    sdsc = np.ascontiguousarray(sds)
    t = time.perf_counter()
    th = L.rsref_run_batch(st.ctypes.data, n, sdsc.ctypes.data, idx.ctypes.data, ctl.ctypes.data, decisions, 0, None)
    dt = time.perf_counter() - t
    return n * decisions * 8 / dt, th, dt


class Clocks:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, index):
        self.index, self.rows, self.p = index, [], None

    def __enter__(self):
        q = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
            "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None
        return self

    def _read(self):
        for line in self.p.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.t.join(timeout=2)

    def summary(self):
        rows = [r for r in self.rows if len(r) >= 7]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][1]) if rows[0][1].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import rsx

    L = oracle_batch()
    if L is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/librsbatch.so not built (the reference sources were absent)"}))
        return
    n = args.arenas
    sample = min(args.cpu_sample, n)
    sds, idx, st = world(rsx, n, 0, args.seed)
    # each step: one decision of a bounded sample of the workload's arenas (rotating through them)
    for w in range(args.warmup):
        lo = (w * sample) % n
        cpu_run(L, rsx, sds, idx[lo:lo + sample], np.ascontiguousarray(st[lo:lo + sample]), 1, args.seed + w)
    tot_ticks, tot_s, threads = 0, 0.0, 0
    for k in range(args.steps):
        lo = ((args.warmup + k) * sample) % n
        part = np.ascontiguousarray(st[lo:lo + sample])
        v, threads, dt = cpu_run(L, rsx, sds, np.ascontiguousarray(idx[lo:lo + sample]), part, 1, args.seed + 100 + k)
        tot_ticks += sample * 8
        tot_s += dt
    value = tot_ticks / tot_s
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "arena-ticks/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_s / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": f"headline mix, {n} arenas, 7x7 car pairings; each step one decision of a {sample}-arena sample",
                                         "arenas": n, "sample_arenas": sample},
        "cpu_baseline": {"value": value, "unit": "arena-ticks/s", "cores": threads, "kind": "reference",
                         "sample": f"{sample} arenas x 1 decision per step, {args.steps} steps"},
        "e2e": {"value": value, "unit": "arena-ticks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_ours(args):
    import torch
    import rsx

    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = rsx.SimDevice(local)
    n = args.arenas
    sds, idx, st = world(rsx, n, rank, args.seed)
    dsd = dev.upload_static(sds)
    ds = dev.upload_states(st)
    didx = torch.from_numpy(idx).to(dev.device)
    steps = args.warmup + args.steps
    ctl_host = np.stack([rsx.decision_controls(args.seed * 1000 + rank, s, n) for s in range(steps)])  # (steps, n, 16)
    dctl = torch.from_numpy(ctl_host.view(np.int32)).to(dev.device)
    res = dev.alloc_result(n)
    ev = torch.zeros(n, dtype=torch.int32, device=dev.device)
    stream = torch.cuda.Stream(device=dev.device)  # every launch and copy of the run goes on this stream
    sptr = stream.cuda_stream
    counter = torch.zeros(1, dtype=torch.int32, device=dev.device)
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    launches_per_step = 1 if args.mode == "plain" else 2  # the persistent path clears its queue counter first

    def step(s, controls_ptr):
        if args.mode == "plain":
            rc = rsx.lib().rsx_sim8_multi_raw(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), controls_ptr, res.data_ptr(), ev.data_ptr(), args.block,
                                              sptr)
        else:
            rc = rsx.lib().rsx_sim8_persistent_raw(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), controls_ptr, res.data_ptr(), ev.data_ptr(), None,
                                                   counter.data_ptr(), sms * 4, args.block, 1, sptr)
        rsx.check(rc, "decision")

    def barrier():
        if dist:
            dist.barrier()

    torch.cuda.synchronize()
    # ---- device-resident timing (value) ----
    for s in range(args.warmup):
        step(s, dctl[s].data_ptr())
    stream.synchronize()
    barrier()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with Clocks(local) as clk:
        evs[0].record(stream)
        for k in range(args.steps):
            step(args.warmup + k, dctl[args.warmup + k].data_ptr())
            evs[k + 1].record(stream)
        evs[-1].synchronize()
    barrier()
    ms_steps = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    t_ms = sum(ms_steps)
    if dist:
        tt = torch.tensor([t_ms], device=dev.device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_ms = float(tt.item())
    value = world_size * n * 8 * args.steps / (t_ms / 1e3)

    # ---- end to end through the public entry point: pinned host controls in, result words out, every step ----
    pin_ctl = torch.from_numpy(ctl_host.view(np.int32)).pin_memory()
    pin_res = torch.zeros(n, dtype=torch.int32).pin_memory()
    dctl1 = torch.zeros((n, 16), dtype=torch.int32, device=dev.device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        for s in range(2):
            dctl1.copy_(pin_ctl[s], non_blocking=True)
            step(s, dctl1.data_ptr())
            pin_res.copy_(res, non_blocking=True)
        stream.synchronize()
        barrier()
        e0.record(stream)
        for k in range(args.steps):
            dctl1.copy_(pin_ctl[args.warmup + k], non_blocking=True)
            step(args.warmup + k, dctl1.data_ptr())
            pin_res.copy_(res, non_blocking=True)
            stream.synchronize()  # the caller reads the step's result words
        e1.record(stream)
        e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if dist:
        tt = torch.tensor([e2e_ms], device=dev.device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_ms = float(tt.item())
    e2e = world_size * n * 8 * args.steps / (e2e_ms / 1e3)
    r = pin_res.numpy().view(np.uint32)
    flags = {"scored": int(((r & 0xFF) != 0).sum()), "overflow": int(((r >> 30) & 1).sum()), "unimplemented": int((r >> 31).sum())}

    # ---- roofline of the decision kernel (HBM: algorithmic bytes per launch / launch time) ----
    mean_ms = t_ms / args.steps
    alg_bytes = n * 8 * ALG_BYTES_PER_ARENA_TICK
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg_bytes / (mean_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms_per_launch": mean_ms}

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        L = oracle_batch()
        if L is not None:
            sample = min(args.cpu_sample, n)
            part = np.ascontiguousarray(st[:sample])
            v, th, dt = cpu_run(L, rsx, sds, np.ascontiguousarray(idx[:sample]), part, 2, 77)
            cpu = {"value": v, "unit": "arena-ticks/s", "cores": th, "kind": "reference",
                   "sample": f"{sample} arenas x 2 decisions of the headline workload ({dt:.1f} s)"}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "arena-ticks/s", "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded states and arena mesh)",
            "config": {"workload": "headline: 65,536 arenas per GPU, mixed states, 7x7 car pairings, one 8-tick decision per step",
                       "arenas_per_gpu": n, "mode": args.mode, "block": args.block,
                       "l2": "inputs larger than L2 (AoSoA state buffer 730 MB per GPU)", "parallelism": f"replicas x{world_size}"},
            "e2e": {"value": e2e, "unit": "arena-ticks/s", "h2d_bytes_per_step": n * 64, "d2h_bytes_per_step": n * 4},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": launches_per_step * args.steps,
            "result_flags": flags,
            "ms_per_step_all": ms_steps,
        }))
    torch.cuda.synchronize()
    ds.free()
    dsd.free()
    if dist:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
