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
TRAFFIC_PER_ARENA_DECISION = 4.716e9 / 32768
# k_observe: 103 state words always read (ball 9, tick 2, the 34 pads' "gave boost" flags, both cars' 29; a pad's tick
# words only when its flag is set), result + event OR + pairing index 9 bytes, two 208-byte FP16 rows and two FP32
# rewards written
OBS_BYTES_PER_ARENA = 103 * 4 + 9 + 2 * 208 + 2 * 4
OBS_REPS = 20
# instruction counts of the lockstep kernel (block 448, split 7) from the same ncu capture as the traffic: 740.69 M warp
# instructions with 7.79 of 32 lanes active on average for one 32,768-arena decision (8 ticks)
WARP_INST_PER_ARENA_TICK = 740.69e6 / (32768 * 8)
LANES_ACTIVE = 7.79
PRESETS = [(p, q) for p in range(7) for q in range(7)]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--arenas", type=int, default=ARENAS)
    ap.add_argument("--mode", default="binned", choices=["plain", "lockstep", "binned"],
                    help="binned: autotuned lockstep kernel with the learned binning among its candidates")
    ap.add_argument("--threshold", type=float, default=0.5, help="binned without the autotuner: predicted-contact threshold")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="launch the timed decisions one by one instead of as CUDA graphs")
    ap.add_argument("--train-decisions", type=int, default=32, help="decisions of exact labels for the predictor")
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--block", type=int, default=448, help="threads per block of the lockstep kernel")
    ap.add_argument("--grid", type=int, default=0, help="lockstep blocks (0: one per SM)")
    ap.add_argument("--split", type=int, default=6,
                    help="lockstep barriers: 0 per phase, 1 + per car in P1, 2 + P1 in parts, 3 + per P3b step, 6 = 2 + P5 and P8 in parts")
    ap.add_argument("--plain-block", type=int, default=32, help="threads per block of the plain launch (the reference's SIM8_BLOCK)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain launch's comparison timing")
    ap.add_argument("--cpu-sample", type=int, default=0, help="reference arm: arenas per step (0: all)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline: seconds of decisions of the workload")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-clocks", action="store_true", help="do not sample nvidia-smi during the timed region")
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


def cpu_run(L, rsx, sds, idx, st, decisions, seed, first=0):
    """The reference's CPU build over `st` (in place) for `decisions` decisions (controls of decisions first,
    first + 1, ... of `seed`) on all host threads; returns (arena-ticks/s, threads, seconds)."""
    n = st.shape[0]
    ctl = np.ascontiguousarray(np.stack([rsx.decision_controls(seed, first + d, n) for d in range(decisions)]))
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
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "50"],
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
    sample = n if args.cpu_sample <= 0 else min(args.cpu_sample, n)
    sds, idx, st = world(rsx, n, 0, args.seed)
    st = np.ascontiguousarray(st[:sample])
    idx = np.ascontiguousarray(idx[:sample])
    # step s: one decision of the (sampled) workload with the controls the GPU arm uses for its step s
    for w in range(args.warmup):
        cpu_run(L, rsx, sds, idx, st, 1, args.seed * 1000, first=w)
    tot_ticks, tot_s, threads = 0, 0.0, 0
    for k in range(args.steps):
        _, threads, dt = cpu_run(L, rsx, sds, idx, st, 1, args.seed * 1000, first=args.warmup + k)
        tot_ticks += sample * 8
        tot_s += dt
    value = tot_ticks / tot_s
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "arena-ticks/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_s / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": f"headline mix, {n} arenas, 7x7 car pairings; each step one decision of {sample} of them",
                                         "arenas": n, "sample_arenas": sample},
        "cpu_baseline": {"value": value, "unit": "arena-ticks/s", "cores": threads, "kind": "reference",
                         "sample": f"{sample} arenas x 1 decision per step, {args.steps} steps ({tot_s:.1f} s)"},
        "e2e": {"value": value, "unit": "arena-ticks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_ours(args):
    import torch
    import rsx
    import predictor as P
    import replicas
    from runner import DecisionRunner

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
    run = DecisionRunner(dev, sds, idx, st)
    stream = run.stream
    steps = args.warmup + args.steps
    ctl_host = np.stack([rsx.decision_controls(args.seed * 1000 + rank, s, n) for s in range(steps)])  # (steps, n, 16)
    dctl = torch.from_numpy(ctl_host.view(np.int32)).to(dev.device)
    torch.cuda.synchronize()
    start = run.snapshot()

    def barrier():
        if dist:
            dist.barrier()

    def reduce_max(x):
        return replicas.max_over_ranks(x, dist, dev.device)

    def timed(config, graph=False, clk=None):
        """W warm-up + K timed decisions of `config` from the start states; (device ms of the K, per-step ms)."""
        run.restore(start)
        for s in range(args.warmup):
            run.step(dctl[s].data_ptr(), config)
        graphs = []
        if graph:  # the K timed decisions as CUDA graphs of up to 16 decisions (captured, not run, here)
            for g0 in range(0, args.steps, 16):
                ptrs = [dctl[args.warmup + k].data_ptr() for k in range(g0, min(args.steps, g0 + 16))]
                graphs.append((len(ptrs), run.capture(ptrs, config)))
        stream.synchronize()
        barrier()
        if clk:
            clk.__enter__()
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        evs[0].record(stream)
        if graph:
            k = 0
            for cnt, g in graphs:
                run.replay(g)
                k += cnt
                evs[k].record(stream)
        else:
            for k in range(args.steps):
                run.step(dctl[args.warmup + k].data_ptr(), config)
                evs[k + 1].record(stream)
        evs[-1].synchronize()
        if clk:
            clk.__exit__()
        barrier()
        if graph:  # one time per graph
            marks = [0] + list(np.cumsum([cnt for cnt, _ in graphs]))
            ms = [evs[marks[i]].elapsed_time(evs[marks[i + 1]]) for i in range(len(graphs))]
        else:
            ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
        t = evs[0].elapsed_time(evs[-1])
        del graphs
        return reduce_max(t), ms

    # ---- the learned part: labels from exact decisions (their own controls), then training ----
    pred_info = None
    if args.mode == "binned":
        t0 = time.perf_counter()
        samples, losses = run.train_predictor(args.seed * 1000 + 500 + rank, decisions=args.train_decisions, epochs=args.epochs)
        pred_info = {"train_samples": samples, "train_seconds": time.perf_counter() - t0, "last_losses": losses}

    # ---- the autotuner: every candidate on the same 2 decisions from the same start states ----
    tune_ctl = [torch.from_numpy(rsx.decision_controls(args.seed * 1000 + 700 + rank, d, n).view(np.int32)).to(dev.device) for d in range(2)]
    torch.cuda.synchronize()
    if args.mode in ("binned", "lockstep") and not args.no_tune:
        # tuned on the states the timed decisions start from (after the warm-up decisions), with controls of their own
        run.restore(start)
        for s_ in range(args.warmup):
            run.step(dctl[s_].data_ptr(), {"mode": "plain", "block": args.plain_block})
        cands = run.candidates(binning=args.mode == "binned")
        tuned = run.tune([c.data_ptr() for c in tune_ctl], cands, repeats=2)
        config = dict(run.config)
        tune_top = [{"ms": round(ms, 3), **c} for ms, c in tuned[:6]]
    elif args.mode == "plain":
        config = {"mode": "plain", "block": args.plain_block}
        tune_top = None
    else:
        config = {"mode": args.mode, "block": args.block, "grid": args.grid or run.sms, "split": args.split, "threshold": args.threshold}
        tune_top = None
    config = replicas.broadcast_config(config, dist, dev.device)  # every rank runs rank 0's configuration

    # ---- timing: the plain launch, the best unbinned lockstep, then the chosen configuration ----
    modes = {}
    if not args.no_plain and config["mode"] != "plain":
        t_plain, _ = timed({"mode": "plain", "block": args.plain_block})
        modes["plain"] = world_size * n * 8 * args.steps / (t_plain / 1e3)
    if config["mode"] in ("binned", "levels") and tune_top:
        unb = next((c for c in [dict(c) for _, c in tuned] if c["mode"] == "lockstep"), None)
        if unb:
            t_unb, _ = timed(unb, graph=not args.no_graph)
            modes["lockstep_unbinned"] = world_size * n * 8 * args.steps / (t_unb / 1e3)
    clk = Clocks(local)
    t_ms, ms_steps = timed(config, graph=not args.no_graph and config["mode"] != "plain", clk=None if args.no_clocks else clk)
    value = world_size * n * 8 * args.steps / (t_ms / 1e3)
    modes[config["mode"]] = value
    words_tuned = run.snapshot()

    # ---- bit-exactness of the chosen configuration against the plain launch (same decisions, same start states) ----
    exact = None
    if not args.no_plain and config["mode"] != "plain":
        timed({"mode": "plain", "block": args.plain_block})
        a = torch.equal(run.snapshot(), words_tuned)
        exact = bool(a)

    # ---- recall / precision of the predictor on the timed decisions ----
    if pred_info is not None:
        run.restore(start)
        Zs, Ys = [], []
        with torch.cuda.stream(stream):  # the copies on the stream the kernels wrote on
            for s in range(steps):
                cp = dctl[s].data_ptr()
                run.step(cp, {"mode": "binned", "block": 448, "grid": run.sms, "split": 7, "threshold": 0.5})
                Zs.append(run.Z.clone())
                Ys.append(run.pred.labels(run.ev.data_ptr(), n).clone())
        stream.synchronize()
        m = P.recall_precision(torch.cat(Zs).cpu().numpy(), torch.cat(Ys).cpu().numpy())
        pred_info["recall_precision_rate"] = {k: [round(float(x), 4) for x in v] for k, v in m.items()}
        pred_info["eval"] = f"{steps} decisions x {n} arenas (the bench's own decisions), threshold 0.5"

    # ---- end to end through the public entry point: pinned host controls in, result words out, every step ----
    pin_ctl = torch.from_numpy(ctl_host.view(np.int32)).pin_memory()
    pin_res = torch.zeros(n, dtype=torch.int32).pin_memory()
    dctl1 = torch.zeros((n, 16), dtype=torch.int32, device=dev.device)
    run.restore(start)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        for s in range(args.warmup):
            dctl1.copy_(pin_ctl[s], non_blocking=True)
            run.step(dctl1.data_ptr(), config)
            pin_res.copy_(run.res, non_blocking=True)
        stream.synchronize()
        barrier()
        e0.record(stream)
        for k in range(args.steps):
            dctl1.copy_(pin_ctl[args.warmup + k], non_blocking=True)
            run.step(dctl1.data_ptr(), config)
            pin_res.copy_(run.res, non_blocking=True)
            stream.synchronize()  # the caller reads the step's result words
        e1.record(stream)
        e1.synchronize()
    e2e_ms = reduce_max(e0.elapsed_time(e1))
    e2e = world_size * n * 8 * args.steps / (e2e_ms / 1e3)
    r = pin_res.numpy().view(np.uint32)
    flags = {"scored": int(((r & 0xFF) != 0).sum()), "overflow": int(((r >> 30) & 1).sum()), "unimplemented": int((r >> 31).sum())}

    # ---- observations and rewards after the decision (k_observe), timed alone on the same states ----
    weights = [10.0, 0.5, 0.25, 2.0, -2.0, 0.125, 0.01, 0.02]
    with torch.cuda.stream(stream):
        for _ in range(3):
            run.observe(weights)
        o0, o1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        o0.record(stream)
        for _ in range(OBS_REPS):
            run.observe(weights)
        o1.record(stream)
        o1.synchronize()
    obs_ms = reduce_max(o0.elapsed_time(o1)) / OBS_REPS

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
    # DRAM bytes (read + write) per arena-decision of the lockstep kernel (block 448, split 7), from one ncu capture
    # (dram__bytes_read.sum + dram__bytes_write.sum: 4.716 GB for one 32,768-arena decision), scaled by the arena count
    traffic = TRAFFIC_PER_ARENA_DECISION * n if config["mode"] != "plain" else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum, scaled from 32,768 arenas)",
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms_per_launch": mean_ms}

    # the second roofline: instruction issue (4 schedulers per SM issue one warp instruction per cycle each)
    sms = torch.cuda.get_device_properties(dev.device).multi_processor_count
    clk_hz = float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
    warp_issue_peak = sms * 4 * clk_hz
    per_gpu = value / world_size
    roofline_issue = {"bound": "issue", "unit": "warp instructions/s",
                      "achieved": WARP_INST_PER_ARENA_TICK * per_gpu, "peak": warp_issue_peak,
                      "frac": WARP_INST_PER_ARENA_TICK * per_gpu / warp_issue_peak,
                      "simt_efficiency": LANES_ACTIVE / 32.0,
                      "thread_instruction_frac": WARP_INST_PER_ARENA_TICK * LANES_ACTIVE * per_gpu / (warp_issue_peak * 32),
                      "per_arena_tick": {"warp_instructions": WARP_INST_PER_ARENA_TICK, "lanes_active": LANES_ACTIVE},
                      "source": "ncu capture of k_sim8_lockstep_t448<7> at 32,768 arenas (instructions per arena-tick), sm_max_mhz"} \
        if config["mode"] != "plain" else None
    observe = {"kernel": "k_observe", "ms_per_launch": obs_ms, "arenas": n,
               "achieved_gbs": OBS_BYTES_PER_ARENA * n / (obs_ms / 1e3) / 1e9,
               "frac": OBS_BYTES_PER_ARENA * n / (obs_ms / 1e3) / 1e9 / peak, "bytes_per_arena": OBS_BYTES_PER_ARENA,
               "share_of_decision": obs_ms / mean_ms}

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        L = oracle_batch()
        if L is not None:
            # decisions of the whole workload from its start states until about cpu_seconds of CPU time have passed
            part = np.ascontiguousarray(st)
            ticks, secs, d, th = 0, 0.0, 0, 0
            while secs < args.cpu_seconds or d < 2:
                _, th, dt = cpu_run(L, rsx, sds, idx, part, 1, args.seed * 1000, first=d)
                ticks += n * 8
                secs += dt
                d += 1
            cpu = {"value": ticks / secs, "unit": "arena-ticks/s", "cores": th, "kind": "reference",
                   "sample": f"{n} arenas x {d} decisions of the same workload from its start states ({secs:.1f} s)"}
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "arena-ticks/s", "n_gpus": world_size, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded states and arena mesh)",
            "config": {"workload": f"headline: {n} arenas per GPU, mixed states, 7x7 car pairings, one 8-tick decision per step",
                       "arenas_per_gpu": n, **config, "cuda_graphs": (not args.no_graph and config["mode"] != "plain"),
                       "l2": f"inputs larger than L2 (AoSoA state buffer {rsx.aosoa_words(n) * 4 / 1e6:.0f} MB per GPU)",
                       "parallelism": f"replicas x{world_size}"},
            "modes": modes,
            "speedup_vs_plain": value / modes["plain"] if "plain" in modes else None,
            "bit_exact_vs_plain": exact,
            "autotune_top": tune_top,
            "predictor": pred_info,
            "e2e": {"value": e2e, "unit": "arena-ticks/s", "h2d_bytes_per_step": n * 64, "d2h_bytes_per_step": n * 4},
            "roofline": roofline,
            "roofline_issue": roofline_issue,
            "observe": observe,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": run.kernels_per_step(config) * args.steps,
            "result_flags": flags,
            "ms_per_step_all": ms_steps,
        }))
    torch.cuda.synchronize()
    run.free()
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
