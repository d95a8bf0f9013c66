#!/usr/bin/env python
"""Benchmark of the soccar 1v1 8-tick decision step on B200.

Metric: arena-ticks/s of one 8-tick decision over 65,536 arenas per GPU (the headline configuration: mixed start
states 20% kickoff / 50% open play / 15% head-on / 10% pinch / 5% pad contention, car pairings uniform over the 7 x 7
hitbox presets, random controls held for 8 ticks), bit-exact with the reference's CPU build.  A step is one decision of
every arena.  Seeded synthetic states over a seeded synthetic arena stand in for the reference's V3-played states and
the game's meshes (neither exists here).

  python bench.py [--gpus N --steps K --warmup W]          this implementation (one JSON line)
  python bench.py --impl reference ...                     the reference's own CPU build on the host's cores (and, for
                                                           context, the reference's own GPU kernel sim8 on this GPU)
  python bench.py --sweep [--sizes 4096,...,1048576]       the arena-count sweep (one JSON line per size)
  python bench.py --zones [--zones-all] [--mix contact]    zone-timer profile of one decision (librsx_zones*.so)
  python bench.py --profile-variants                       one decision of each decision kernel, for an ncu capture

`value` is device time of the decision kernels with states resident in HBM (max over ranks); `e2e` times the public
entry point with the controls copied from pinned host memory and the result words read back every step.  After the
timing, every arena of every timed decision is replayed through the oracle (the reference's CPU build) and compared word
for word (`bit_exact_vs_oracle`); a second leg repeats plain vs tuned at 262,144 arenas with a 1% oracle sample.
N > 1: one process per GPU, each with its own arenas (weak scaling); arenas are independent, so no collective touches
the data path (the timing max is the only reduction).
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
LARGE_ARENAS = 262144
TICK_WORDS = 2567
TICK_BYTES = TICK_WORDS * 4
ALG_BYTES_PER_ARENA_TICK = (TICK_BYTES * 2 + 64 + 4) / 8.0  # state in + out, controls, result, per tick
METRIC = "arena-ticks/s, 8-tick decision, 65,536 arenas: binned vs plain, bit-exact"
# k_observe: 103 state words always read (ball 9, tick 2, the 34 pads' "gave boost" flags, both cars' 29; a pad's tick
# words only when its flag is set), result + event OR + pairing index 9 bytes, two 208-byte FP16 rows and two FP32
# rewards written
OBS_BYTES_PER_ARENA = 103 * 4 + 9 + 2 * 208 + 2 * 4
OBS_REPS = 20
PRESETS = [(p, q) for p in range(7) for q in range(7)]

# Per decision-kernel counters of one 65,536-arena headline decision from one ncu capture of all variants (the third
# decision of each after 8 decisions of the plain launch from the start states, as `bench.py --profile-variants` runs
# them: the contact-richer states the timed decisions see; dram__bytes_read.sum + dram__bytes_write.sum,
# smsp__inst_executed.sum, smsp__thread_inst_executed.sum; the command is in profiles/k_sim8_lockstep_headline.md):
# DRAM bytes per arena-decision, warp instructions per arena-tick, lanes active per warp instruction.
_N, _T = 65536, 65536 * 8


def _kc(rd, wr, inst, thr):
    return {"dram_bytes_per_arena": (rd + wr) / _N, "warp_inst_per_arena_tick": inst / _T, "lanes_active": thr / inst,
            "capture": "65,536 arenas, a headline decision after 8 (same size as the timed run)"}


KERNEL_COUNTERS = {
    "k_sim8_multi": _kc(5126267136, 5056344576, 1534066674, 10436083984),
    "k_sim8_lockstep_t448<7>": _kc(6258553856, 5842978816, 1551714381, 10758340571),
    "k_sim8_lockstep_t512<7>": _kc(6255863552, 5833099776, 1552293325, 10775763619),
    "k_sim8_lockstep_t448<14>": _kc(5870563840, 5579853312, 1213356967, 11506029617),
    "k_sim8_lockstep_t512<14>": _kc(5894772480, 5602215168, 1217023574, 11597969422),
    "k_sim8_lockstep_t448<15>": _kc(5848313600, 5567679232, 1167464173, 11751954768),
    "k_sim8_lockstep_t512<15>": _kc(5877518848, 5585444608, 1172608364, 11849352609),
}


def kernel_name(config):
    m = config["mode"]
    if m == "plain":
        return "k_sim8_multi"
    if m == "sim8":
        return "k_sim8"
    if m == "persistent":
        return f"k_sim8_persistent_b{config['min_blocks']}"
    t = 448 if config["block"] <= 448 else 512
    name = f"k_sim8_lockstep_t{t}<{config['split']}>"
    return name if config.get("ticks", 8) == 8 else f"{name} x{8 // config['ticks']} launches"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--arenas", type=int, default=ARENAS)
    ap.add_argument("--large-arenas", type=int, default=LARGE_ARENAS, help="arenas of the second leg (0: none)")
    ap.add_argument("--large-steps", type=int, default=8, help="timed decisions of the second leg")
    ap.add_argument("--mode", default="binned", choices=["plain", "lockstep", "binned"],
                    help="binned: autotuned lockstep kernel with the learned binning among its candidates")
    ap.add_argument("--threshold", type=float, default=0.5, help="binned without the autotuner: predicted-contact threshold")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--tune-decisions", type=int, default=4)
    ap.add_argument("--tune-repeats", type=int, default=3)
    ap.add_argument("--no-graph", action="store_true", help="launch the timed decisions one by one instead of as CUDA graphs")
    ap.add_argument("--train-decisions", type=int, default=32, help="decisions of exact labels for the predictor")
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--block", type=int, default=448, help="threads per block of the lockstep kernel")
    ap.add_argument("--grid", type=int, default=0, help="lockstep blocks (0: one per SM)")
    ap.add_argument("--split", type=int, default=15,
                    help="lockstep barriers: 0 per phase, 1 + per car in P1, 2 + P1 in parts, 3 + per P3b step, 6 = 2 + P5 and P8 in parts, "
                         "7 = 6 + P3a per body, 9 = 7 + P3b's leaf tests pooled over the block, 10 = 9 + the wheel rays' mesh leaves pooled")
    ap.add_argument("--plain-block", type=int, default=32, help="threads per block of the plain launch (the reference's SIM8_BLOCK)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain launch's comparison timing")
    ap.add_argument("--no-oracle", action="store_true", help="skip the word-for-word replay through the oracle")
    ap.add_argument("--no-context", action="store_true", help="skip the one-pairing leg timed beside the reference's GPU kernel")
    ap.add_argument("--cpu-sample", type=int, default=0, help="reference arm: arenas per step (0: all)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU baseline: seconds of decisions of the workload")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-clocks", action="store_true", help="do not sample nvidia-smi during the timed region")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--sweep", action="store_true", help="the arena-count sweep instead of the bench line")
    ap.add_argument("--sizes", default="4096,16384,65536,262144,1048576")
    ap.add_argument("--sweep-decisions", type=int, default=4)
    ap.add_argument("--zones", action="store_true", help="zone-timer profile instead of the bench line")
    ap.add_argument("--zones-all", action="store_true", help="with --zones: every marker of the simulator")
    ap.add_argument("--zones-lockstep", action="store_true", help="with --zones: the pieces of the lockstep kernel at --split (block 448)")
    ap.add_argument("--zones-skip", type=int, default=0, help="with --zones: plain decisions run first (untimed)")
    ap.add_argument("--mix", default="headline", choices=["headline", "contact"])
    ap.add_argument("--rollout", action="store_true",
                    help="the on-device rollout (1,048,576 arenas, contact-heavy mix, 1,000 decisions, retraining, resets) with "
                         "a 1%% sample checked against the oracle at decisions 1, 500 and 1,000")
    ap.add_argument("--rollout-arenas", type=int, default=1048576)
    ap.add_argument("--rollout-decisions", type=int, default=1000)
    ap.add_argument("--profile-variants", action="store_true",
                    help="one decision of the plain launch and of each lockstep variant after two of its own, for an ncu capture")
    return ap.parse_args()


def world(rsx, n, rank, seed, mix=None):
    """The 49 car pairings' StaticData, a pairing per arena, and the mixed start states."""
    sds = np.stack([rsx.build_static(7, p, q) for p, q in PRESETS])
    with np.errstate(over="ignore"):
        h = rsx._mix64(np.arange(n, dtype=np.uint64) + np.uint64((rank + 1) << 40))
    idx = (h % np.uint64(len(PRESETS))).astype(np.uint8)
    st = rsx.make_states_multi(sds, idx, seed + rank, mix or rsx.MIX_HEADLINE)
    return sds, idx, st


def world_one_pairing(rsx, n, seed):
    """The same mixed start states with one car pairing (Octane vs Octane) for every arena: the workload the reference's
    own sim8, which takes one StaticData, runs unchanged."""
    sd = rsx.build_static(7, 0, 0)
    idx = np.zeros(n, np.uint8)
    return sd[None], idx, rsx.make_states_multi(sd[None], idx, seed, rsx.MIX_HEADLINE)


def controls_of(rsx, seed, first, count, n):
    return np.ascontiguousarray(np.stack([rsx.decision_controls(seed, first + d, n) for d in range(count)]))


def oracle_batch():
    path = os.path.join(ROOT, "oracle", "_ref", "librsbatch.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    vp, u32 = ctypes.c_void_p, ctypes.c_uint32
    L.rsref_run_batch.argtypes = [vp, u32, vp, vp, vp, u32, ctypes.c_int, vp]
    if hasattr(L, "rsref_run_batch_ex"):
        L.rsref_run_batch_ex.argtypes = [vp, u32, vp, vp, vp, u32, vp, u32, ctypes.c_int, vp, vp]
    return L


def cpu_run(L, sds, idx, st, ctl):
    """The reference's CPU build over `st` (in place) for the decisions of `ctl` (decisions, n, 16) on all host threads;
    returns (arena-ticks/s, threads, seconds)."""
    n = st.shape[0]
    sdsc = np.ascontiguousarray(sds)
    t = time.perf_counter()
    th = L.rsref_run_batch(st.ctypes.data, n, sdsc.ctypes.data, idx.ctypes.data, ctl.ctypes.data, ctl.shape[0], 0, None)
    dt = time.perf_counter() - t
    return n * ctl.shape[0] * 8 / dt, th, dt


def oracle_compare(L, sds, idx, st0, ctl, sample, got_words, got_res, got_ev):
    """Replays arenas `sample` (indices into the workload) from their start states st0[sample] through the oracle for
    the decisions of `ctl` (decisions, n, 16) and compares, word for word, every decision's result word and event OR
    (got_res / got_ev: (decisions, len(sample)) u32) and the tick-boundary words after the last decision (got_words:
    (len(sample), >= 2567) u32).  Returns the bit_exact_vs_oracle record."""
    m = len(sample)
    d = ctl.shape[0]
    st = np.ascontiguousarray(st0[sample])
    res = np.zeros((d, m), np.uint32)
    ev = np.zeros((d, m), np.uint32)
    smp = np.ascontiguousarray(sample.astype(np.uint32))
    sidx = np.ascontiguousarray(idx[sample])
    t = time.perf_counter()
    sdsc = np.ascontiguousarray(sds)  # referenced until the call returns (a copy when sds is not contiguous)
    L.rsref_run_batch_ex(st.ctypes.data, m, sdsc.ctypes.data, sidx.ctypes.data, ctl.ctypes.data, ctl.shape[1],
                         smp.ctypes.data, d, 0, res.ctypes.data, ev.ctypes.data)
    secs = time.perf_counter() - t
    bad_state = np.any(st[:, :TICK_WORDS] != got_words[:, :TICK_WORDS], axis=1)
    bad_res = np.any(res != got_res, axis=0)
    bad_ev = np.any(ev != got_ev, axis=0)
    bad = bad_state | bad_res | bad_ev
    return {"arenas": int(m), "decisions": int(d), "mismatches": int(bad.sum()), "state_mismatches": int(bad_state.sum()),
            "result_mismatches": int(bad_res.sum()), "event_mismatches": int(bad_ev.sum()),
            "words_compared": int(m * TICK_WORDS + 2 * m * d), "scored": int(((res & 0xFF) != 0).sum()),
            "first_bad": [int(x) for x in sample[np.nonzero(bad)[0][:4]]], "oracle_seconds": round(secs, 2)}


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


# ---------------------------------------------------------------------------------------------------------------------
# the reference arm
# ---------------------------------------------------------------------------------------------------------------------
def reference_gpu_context(args, rsx):
    """The reference's own GPU kernel (cuda/sim/sim.cu sim8, compiled unchanged for sm_100a into oracle/_ref) on this GPU:
    the one-pairing workload, W untimed + K timed decisions, block 32 as the reference's host crate launches it; a 1%
    sample checked word for word against the reference's CPU build.  Context only: not this arm's value."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refgpu

    if not refgpu.available():
        return {"unavailable": "oracle/_ref/sim8_ref.cubin not built (make -C oracle gpu needs the reference's sources)"}
    import torch

    n = args.arenas
    sds, idx, st = world_one_pairing(rsx, n, args.seed)
    ref = refgpu.RefSim8(0)
    stream = torch.cuda.Stream()
    d_states = torch.from_numpy(rsx.pack(st).view(np.int32)).cuda()
    d_sd = torch.from_numpy(np.ascontiguousarray(sds.reshape(-1)).view(np.int32)).cuda()
    steps = args.warmup + args.steps
    ctl = controls_of(rsx, args.seed * 1000, 0, steps, n)
    d_ctl = torch.from_numpy(ctl.view(np.int32)).cuda()
    d_res = torch.zeros(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    for s in range(args.warmup):
        ref.sim8(d_states.data_ptr(), n, d_sd.data_ptr(), d_ctl[s].data_ptr(), d_res.data_ptr(), stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        ref.sim8(d_states.data_ptr(), n, d_sd.data_ptr(), d_ctl[args.warmup + k].data_ptr(), d_res.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    out = {"kernel": "sim8 (cuda/sim/sim.cu:95-104, nvcc 12.9 -gencode arch=compute_100a,code=sm_100a, the build crate's float flags)",
           "value": n * 8 * args.steps / (ms / 1e3), "unit": "arena-ticks/s", "ms_per_step": ms / args.steps, "block": refgpu.SIM8_BLOCK,
           "workload": f"{n} arenas, headline mix, one car pairing (Octane vs Octane); each step one decision of all"}
    L = oracle_batch()
    if L is not None and hasattr(L, "rsref_run_batch_ex"):
        # the reference's GPU kernel against its own CPU build: a 1% sample of the arenas over the W + K decisions
        got = rsx.unpack(d_states.cpu().numpy().view(np.uint32), n)
        rng = np.random.default_rng(args.seed + 11)
        sample = np.sort(rng.choice(n, size=max(1, n // 100), replace=False))
        st0 = world_one_pairing(rsx, n, args.seed)[2]
        m = oracle_compare(L, sds, idx, st0, ctl, sample, got[sample], np.zeros((steps, len(sample)), np.uint32),
                           np.zeros((steps, len(sample)), np.uint32))
        out["gpu_vs_cpu_build"] = {"arenas": m["arenas"], "decisions": m["decisions"], "state_mismatches": m["state_mismatches"],
                                   "compared": "tick-boundary words after the last decision"}
    ref.close()
    return out


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
        cpu_run(L, sds, idx, st, controls_of(rsx, args.seed * 1000, w, 1, n)[:, :sample].copy())
    tot_ticks, tot_s, threads = 0, 0.0, 0
    for k in range(args.steps):
        _, threads, dt = cpu_run(L, sds, idx, st, controls_of(rsx, args.seed * 1000, args.warmup + k, 1, n)[:, :sample].copy())
        tot_ticks += sample * 8
        tot_s += dt
    value = tot_ticks / tot_s
    gpu_ctx = None
    try:
        import torch

        if torch.cuda.is_available() and not args.no_context:
            gpu_ctx = reference_gpu_context(args, rsx)
    except Exception as e:  # context only: the CPU value stands without it
        gpu_ctx = {"unavailable": f"{type(e).__name__}: {e}"}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "arena-ticks/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_s / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": {"workload": f"headline mix, {n} arenas, 7x7 car pairings; each step one decision of {sample} of them",
                                         "arenas": n, "sample_arenas": sample},
        "cpu_baseline": {"value": value, "unit": "arena-ticks/s", "cores": threads, "kind": "reference",
                         "sample": f"{sample} arenas x 1 decision per step, {args.steps} steps ({tot_s:.1f} s)"},
        "e2e": {"value": value, "unit": "arena-ticks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu_sim8": gpu_ctx,
    }))


# ---------------------------------------------------------------------------------------------------------------------
# this implementation
# ---------------------------------------------------------------------------------------------------------------------
class Leg:
    """One workload on one GPU: the runner, its start states, the controls of the W + K decisions, the timing helper."""

    def __init__(self, args, dev, sds, idx, st, ctl_seed, dist=None):
        import torch
        import rsx
        from runner import DecisionRunner

        self.torch, self.args, self.dev, self.dist = torch, args, dev, dist
        self.sds, self.idx = sds, idx
        self.n = st.shape[0]
        self.run = DecisionRunner(dev, sds, idx, st)
        self.steps = args.warmup + args.steps
        self.ctl_host = controls_of(rsx, ctl_seed, 0, self.steps, self.n)  # (steps, n, 16)
        self.dctl = torch.from_numpy(self.ctl_host.view(np.int32)).to(dev.device)
        torch.cuda.synchronize()
        self.start = self.run.snapshot()

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def timed(self, config, steps=None, graph=False, clk=None):
        """W warm-up + K timed decisions of `config` from the start states; (device ms of the K, per-step or per-graph ms)."""
        import replicas

        torch, run, args = self.torch, self.run, self.args
        K = steps or args.steps
        run.restore(self.start)
        for s in range(args.warmup):
            run.step(self.dctl[s].data_ptr(), config)
        graphs = []
        if graph:  # the K timed decisions as CUDA graphs of up to 16 decisions (captured, not run, here)
            for g0 in range(0, K, 16):
                ptrs = [self.dctl[args.warmup + k].data_ptr() for k in range(g0, min(K, g0 + 16))]
                graphs.append((len(ptrs), run.capture(ptrs, config)))
        run.stream.synchronize()
        self.barrier()
        if clk:
            clk.__enter__()
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
        evs[0].record(run.stream)
        if graph:
            k = 0
            for cnt, g in graphs:
                run.replay(g)
                k += cnt
                evs[k].record(run.stream)
        else:
            for k in range(K):
                run.step(self.dctl[args.warmup + k].data_ptr(), config)
                evs[k + 1].record(run.stream)
        evs[-1].synchronize()
        if clk:
            clk.__exit__()
        self.barrier()
        if graph:  # one time per graph
            marks = [0] + list(np.cumsum([cnt for cnt, _ in graphs]))
            ms = [evs[marks[i]].elapsed_time(evs[marks[i + 1]]) for i in range(len(graphs))]
        else:
            ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(K)]
        t = evs[0].elapsed_time(evs[-1])
        del graphs
        return replicas.max_over_ranks(t, self.dist, self.dev.device), ms

    def record_decisions(self, config, steps, sample=None):
        """The W + `steps` decisions of `config` from the start states, one launch sequence per decision, keeping every
        decision's result and event words (of the arenas of `sample`, or all); returns (res, ev) (decisions, m) u32."""
        torch, run = self.torch, self.run
        run.restore(self.start)
        sel = None if sample is None else torch.from_numpy(sample.astype(np.int64)).to(self.dev.device)
        rs, es = [], []
        with torch.cuda.stream(run.stream):
            for s in range(self.args.warmup + steps):
                run.step(self.dctl[s].data_ptr(), config)
                rs.append(run.res.clone() if sel is None else run.res.index_select(0, sel))
                es.append(run.ev.clone() if sel is None else run.ev.index_select(0, sel))
        run.stream.synchronize()
        return torch.stack(rs).cpu().numpy().view(np.uint32), torch.stack(es).cpu().numpy().view(np.uint32)

    def words_of(self, snap, sample=None):
        """Tick-boundary words of the arenas of `sample` (or all) from a device snapshot of the AoSoA buffer."""
        import rsx

        torch = self.torch
        if sample is None:
            return rsx.unpack(snap.cpu().numpy().view(np.uint32), self.n)
        a = torch.from_numpy(sample.astype(np.int64)).to(self.dev.device)[:, None]
        w = torch.arange(TICK_WORDS, device=self.dev.device, dtype=torch.int64)[None, :]
        pos = (a // 32) * (32 * rsx.ARENA_WORDS) + w * 32 + (a % 32)
        return snap[pos.reshape(-1)].reshape(len(sample), TICK_WORDS).cpu().numpy().view(np.uint32)

    def free(self):
        self.run.free()
        del self.start


def tune_leg(leg, args, binning, seed, decisions, repeats):
    """The autotuner over the runner's candidates, on the states the timed decisions start from (after the warm-up
    decisions), with controls of their own; returns (config, top list with spreads)."""
    import rsx

    torch, run = leg.torch, leg.run
    tune_ctl = [torch.from_numpy(rsx.decision_controls(seed, d, leg.n).view(np.int32)).to(leg.dev.device) for d in range(decisions)]
    torch.cuda.synchronize()
    run.restore(leg.start)
    for s_ in range(args.warmup):
        run.step(leg.dctl[s_].data_ptr(), {"mode": "plain", "block": args.plain_block})
    tuned = run.tune([c.data_ptr() for c in tune_ctl], run.candidates(binning=binning), repeats=repeats)
    top = [{"ms_median": round(ms, 3), "ms_best": round(min(ts), 3), "ms_repeats": [round(x, 3) for x in ts], **c} for ms, c, ts in tuned[:8]]
    return dict(run.config), tuned, top


def run_ours(args):
    import torch
    import rsx
    import predictor as P
    import replicas

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
    if args.sweep:
        return sweep(args, dev)
    if args.zones:
        return zones(args, dev)
    if args.rollout:
        return rollout_check(args, dev)
    n = args.arenas
    sds, idx, st = world(rsx, n, rank, args.seed)
    leg = Leg(args, dev, sds, idx, st, args.seed * 1000 + rank, dist)
    run = leg.run
    if args.profile_variants:
        return profile_variants(args, leg)

    # ---- the learned part: labels from exact decisions (their own controls), then training ----
    pred_info = None
    if args.mode == "binned":
        t0 = time.perf_counter()
        samples, losses = run.train_predictor(args.seed * 1000 + 500 + rank, decisions=args.train_decisions, epochs=args.epochs)
        pred_info = {"train_samples": samples, "train_seconds": time.perf_counter() - t0, "last_losses": losses}

    # ---- the autotuner ----
    tuned = None
    if args.mode in ("binned", "lockstep") and not args.no_tune:
        config, tuned, tune_top = tune_leg(leg, args, args.mode == "binned", args.seed * 1000 + 700 + rank, args.tune_decisions,
                                           args.tune_repeats)
    elif args.mode == "plain":
        config, tune_top = {"mode": "plain", "block": args.plain_block}, None
    else:
        config = {"mode": args.mode, "block": args.block, "grid": args.grid or run.sms, "split": args.split, "threshold": args.threshold}
        tune_top = None
    config = replicas.broadcast_config(config, dist, dev.device)  # every rank runs rank 0's configuration

    # ---- timing: the plain launch, the best unbinned lockstep, then the chosen configuration ----
    modes = {}
    graph = not args.no_graph and config["mode"] != "plain"
    if not args.no_plain and config["mode"] != "plain":
        t_plain, _ = leg.timed({"mode": "plain", "block": args.plain_block})
        modes["plain"] = world_size * n * 8 * args.steps / (t_plain / 1e3)
    if config["mode"] in ("binned", "levels") and tuned:
        unb = next((dict(c) for _, c, _ in tuned if c["mode"] == "lockstep"), None)
        if unb:
            t_unb, _ = leg.timed(unb, graph=graph)
            modes["lockstep_unbinned"] = world_size * n * 8 * args.steps / (t_unb / 1e3)
    clk = Clocks(local)
    t_ms, ms_steps = leg.timed(config, graph=graph, clk=None if args.no_clocks else clk)
    value = world_size * n * 8 * args.steps / (t_ms / 1e3)
    modes[config["mode"]] = value
    words_tuned = run.snapshot()

    # ---- bit-exactness of the chosen configuration against the plain launch (same decisions, same start states) ----
    exact = None
    if not args.no_plain and config["mode"] != "plain":
        leg.timed({"mode": "plain", "block": args.plain_block})
        exact = bool(torch.equal(run.snapshot(), words_tuned))

    # ---- every arena of every decision above through the oracle (the reference's CPU build), word for word ----
    vs_oracle = None
    L = oracle_batch()
    if not args.no_oracle and L is not None and hasattr(L, "rsref_run_batch_ex"):
        res_all, ev_all = leg.record_decisions(config, args.steps)
        step_path_same = bool(torch.equal(run.snapshot(), words_tuned))  # the step-by-step replay ends where the graphs did
        vs_oracle = oracle_compare(L, sds, idx, st, leg.ctl_host, np.arange(n), leg.words_of(words_tuned), res_all, ev_all)
        vs_oracle["config"] = kernel_name(config)
        vs_oracle["graph_and_step_paths_equal"] = step_path_same

    # ---- recall / precision of the predictor on the timed decisions ----
    if pred_info is not None:
        run.restore(leg.start)
        Zs, Ys = [], []
        with torch.cuda.stream(run.stream):  # the copies on the stream the kernels wrote on
            for s in range(leg.steps):
                run.step(leg.dctl[s].data_ptr(), {"mode": "binned", "block": 448, "grid": run.sms, "split": 15, "threshold": 0.5})
                Zs.append(run.Z.clone())
                Ys.append(run.pred.labels(run.ev.data_ptr(), n).clone())
        run.stream.synchronize()
        m = P.recall_precision(torch.cat(Zs).cpu().numpy(), torch.cat(Ys).cpu().numpy())
        pred_info["recall_precision_rate"] = {k: [round(float(x), 4) for x in v] for k, v in m.items()}
        pred_info["eval"] = f"{leg.steps} decisions x {n} arenas (the bench's own decisions), threshold 0.5"
        if "lockstep_unbinned" in modes:
            pred_info["learned_order_gain_vs_unbinned"] = value / modes["lockstep_unbinned"]

    # ---- end to end through the public entry point: pinned host controls in, result words out, every step ----
    pin_ctl = torch.from_numpy(leg.ctl_host.view(np.int32)).pin_memory()
    pin_res = torch.zeros(n, dtype=torch.int32).pin_memory()
    dctl1 = torch.zeros((n, 16), dtype=torch.int32, device=dev.device)
    run.restore(leg.start)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(run.stream):
        for s in range(args.warmup):
            dctl1.copy_(pin_ctl[s], non_blocking=True)
            run.step(dctl1.data_ptr(), config)
            pin_res.copy_(run.res, non_blocking=True)
        run.stream.synchronize()
        leg.barrier()
        e0.record(run.stream)
        for k in range(args.steps):
            dctl1.copy_(pin_ctl[args.warmup + k], non_blocking=True)
            run.step(dctl1.data_ptr(), config)
            pin_res.copy_(run.res, non_blocking=True)
            run.stream.synchronize()  # the caller reads the step's result words
        e1.record(run.stream)
        e1.synchronize()
    e2e_ms = replicas.max_over_ranks(e0.elapsed_time(e1), dist, dev.device)
    e2e = world_size * n * 8 * args.steps / (e2e_ms / 1e3)
    r = pin_res.numpy().view(np.uint32)
    flags = {"scored": int(((r & 0xFF) != 0).sum()), "overflow": int(((r >> 30) & 1).sum()), "unimplemented": int((r >> 31).sum())}

    # ---- observations and rewards after the decision (k_observe), timed alone on the same states ----
    weights = [10.0, 0.5, 0.25, 2.0, -2.0, 0.125, 0.01, 0.02]
    with torch.cuda.stream(run.stream):
        for _ in range(3):
            run.observe(weights)
        o0, o1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        o0.record(run.stream)
        for _ in range(OBS_REPS):
            run.observe(weights)
        o1.record(run.stream)
        o1.synchronize()
    obs_ms = replicas.max_over_ranks(o0.elapsed_time(o1), dist, dev.device) / OBS_REPS

    # ---- roofline of the decision kernel (HBM: algorithmic bytes per launch / launch time) ----
    mean_ms = t_ms / args.steps
    launches = 8 // config.get("ticks", 8) if config["mode"] in ("lockstep", "binned", "levels") else 1
    # state in and out, controls and result words once per launch of the decision
    alg_bytes = n * launches * (2 * TICK_BYTES + 64 + 4)
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg_bytes / (mean_ms / 1e3) / 1e9
    kname = kernel_name(config)
    kc = KERNEL_COUNTERS.get(kname)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": kc["dram_bytes_per_arena"] * n if kc else None,
                "traffic_unit": f"bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum of {kname}, {kc['capture']})" if kc else
                f"no ncu capture of {kname} in profiles/",
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback", "kernel": kname,
                "algorithmic_bytes_per_decision": alg_bytes, "launches_per_decision": launches, "kernel_ms_per_decision": mean_ms}
    sms = torch.cuda.get_device_properties(dev.device).multi_processor_count
    clk_hz = float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
    warp_issue_peak = sms * 4 * clk_hz  # 4 schedulers per SM issue one warp instruction per cycle each
    per_gpu = value / world_size
    roofline_issue = None
    if kc:
        wi = kc["warp_inst_per_arena_tick"]
        roofline_issue = {"bound": "issue", "unit": "warp instructions/s", "kernel": kname, "achieved": wi * per_gpu, "peak": warp_issue_peak,
                          "frac": wi * per_gpu / warp_issue_peak, "simt_efficiency": kc["lanes_active"] / 32.0,
                          "thread_instruction_frac": wi * kc["lanes_active"] * per_gpu / (warp_issue_peak * 32),
                          "per_arena_tick": {"warp_instructions": wi, "lanes_active": kc["lanes_active"]},
                          "source": f"ncu capture of {kname}, {kc['capture']}; peak at sm_max_mhz"}
    observe = {"kernel": "k_observe", "ms_per_launch": obs_ms, "arenas": n,
               "achieved_gbs": OBS_BYTES_PER_ARENA * n / (obs_ms / 1e3) / 1e9,
               "frac": OBS_BYTES_PER_ARENA * n / (obs_ms / 1e3) / 1e9 / peak, "bytes_per_arena": OBS_BYTES_PER_ARENA,
               "share_of_decision": obs_ms / mean_ms}

    # ---- the same comparison on one car pairing (the workload the reference's own GPU sim8 runs in its arm) ----
    context = None
    if not args.no_context and world_size == 1:
        context = one_pairing_leg(args, dev, config, run.pred)

    # ---- the second size: 262,144 arenas, plain vs tuned, with a 1% oracle sample ----
    large = None
    if args.large_arenas and world_size == 1:
        leg.free()
        del words_tuned
        torch.cuda.empty_cache()
        large = large_leg(args, dev, run.pred, L)

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline and L is not None:
        # decisions of the whole workload from its start states until about cpu_seconds of CPU time have passed
        part = np.ascontiguousarray(st)
        ticks, secs, d, th = 0, 0.0, 0, 0
        while secs < args.cpu_seconds or d < 2:
            _, th, dt = cpu_run(L, sds, idx, part, controls_of(rsx, args.seed * 1000, d, 1, n))
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
                       "arenas_per_gpu": n, **config, "cuda_graphs": graph,
                       "l2": f"inputs larger than L2 (AoSoA state buffer {rsx.aosoa_words(n) * 4 / 1e6:.0f} MB per GPU)",
                       "parallelism": f"replicas x{world_size}"},
            "modes": modes,
            "speedup_vs_plain": value / modes["plain"] if "plain" in modes else None,
            "bit_exact_vs_plain": exact,
            "bit_exact_vs_oracle": vs_oracle,
            "size_262144": large,
            "one_pairing_vs_reference_gpu": context,
            "autotune": {"decisions": args.tune_decisions, "repeats": args.tune_repeats, "top": tune_top},
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
    if large is None:
        leg.free()
    if dist:
        dist.destroy_process_group()


def one_pairing_leg(args, dev, config, pred):
    """The headline mix with one car pairing for every arena: this project's reference-shaped sim8 entry (k_sim8, block
    32) and the tuned configuration, W + K decisions each; the reference arm times the reference's own sim8 on the same
    states and controls."""
    import rsx

    sds, idx, st = world_one_pairing(rsx, args.arenas, args.seed)
    leg = Leg(args, dev, sds, idx, st, args.seed * 1000)
    leg.run.use_predictor(pred)
    out = {"workload": f"{args.arenas} arenas, headline mix, Octane vs Octane for every arena"}
    t, _ = leg.timed({"mode": "sim8", "block": 32})
    w_sim8 = leg.run.snapshot()
    out["sim8"] = args.arenas * 8 * args.steps / (t / 1e3)
    cfg = dict(config)
    t, _ = leg.timed(cfg, graph=not args.no_graph and cfg["mode"] != "plain")
    out["tuned"] = args.arenas * 8 * args.steps / (t / 1e3)
    out["tuned_config"] = kernel_name(cfg)
    out["same_words"] = bool(leg.torch.equal(leg.run.snapshot(), w_sim8))
    del w_sim8
    leg.free()
    return out


def large_leg(args, dev, pred, L):
    """262,144 arenas of the headline workload: the autotuner at this size (2 decisions, best of 2), the plain launch and
    the tuned configuration timed over W + large_steps decisions from the same start states, all words compared between
    them, and a seeded 1% sample of the arenas replayed through the oracle over every decision."""
    import torch
    import rsx

    n = args.large_arenas
    a2 = argparse.Namespace(**vars(args))
    a2.steps = args.large_steps
    sds, idx, st = world(rsx, n, 0, args.seed + 100)
    leg = Leg(a2, dev, sds, idx, st, args.seed * 1000 + 900)
    leg.run.use_predictor(pred)
    out = {"arenas": n, "steps": a2.steps, "warmup": a2.warmup}
    config, tuned, top = tune_leg(leg, a2, pred is not None, args.seed * 1000 + 950, 2, 2)
    out["autotune_top"] = top[:4]
    graph = not args.no_graph and config["mode"] != "plain"
    t_plain, _ = leg.timed({"mode": "plain", "block": args.plain_block})
    w_plain = leg.run.snapshot()
    out["plain"] = n * 8 * a2.steps / (t_plain / 1e3)
    if config["mode"] in ("binned", "levels"):
        unb = next((dict(c) for _, c, _ in tuned if c["mode"] == "lockstep"), None)
        if unb:
            t_unb, _ = leg.timed(unb, graph=graph)
            out["lockstep_unbinned"] = n * 8 * a2.steps / (t_unb / 1e3)
    t_ms, _ = leg.timed(config, graph=graph)
    out["tuned"] = n * 8 * a2.steps / (t_ms / 1e3)
    out["tuned_config"] = {"kernel": kernel_name(config), **config}
    out["speedup_vs_plain"] = out["tuned"] / out["plain"]
    words = leg.run.snapshot()
    out["bit_exact_vs_plain"] = bool(torch.equal(words, w_plain))
    del w_plain
    if L is not None and hasattr(L, "rsref_run_batch_ex") and not args.no_oracle:
        rng = np.random.default_rng(args.seed + 262144)
        sample = np.sort(rng.choice(n, size=n // 100, replace=False))
        res, ev = leg.record_decisions(config, a2.steps, sample)
        out["bit_exact_vs_oracle"] = oracle_compare(L, sds, idx, st, leg.ctl_host, sample, leg.words_of(words, sample), res, ev)
    del words
    leg.free()
    return out


def profile_variants(args, leg):
    """For ncu captures at the headline size: 8 decisions of the plain launch from the start states (the states the bench
    times are later, contact-richer ones), then for the plain launch and each lockstep variant the autotuner considers
    (blocks 448 / 512, splits 7 / 14 / 15), two decisions and then a third, each from those states.
    Launch order: k_sim8_multi x 8, then 3 launches per variant in the order printed."""
    variants = [{"mode": "plain", "block": 32}] + [{"mode": "lockstep", "block": b, "grid": leg.run.sms, "split": s}
                                                   for b in (448, 512) for s in (7, 14, 15)]
    run = leg.run
    run.restore(leg.start)
    for s in range(8):
        run.step(leg.dctl[s % leg.steps].data_ptr(), {"mode": "plain", "block": 32})
    warm = run.snapshot()
    out = []
    for cfg in variants:
        run.restore(warm)
        e0, e1 = leg.torch.cuda.Event(enable_timing=True), leg.torch.cuda.Event(enable_timing=True)
        for s in range(3):
            if s == 2:
                e0.record(run.stream)
            run.step(leg.dctl[(8 + s) % leg.steps].data_ptr(), cfg)
        e1.record(run.stream)
        e1.synchronize()
        out.append({"kernel": kernel_name(cfg), "ms": e0.elapsed_time(e1)})
    print(json.dumps({"profile_variants": out, "arenas": leg.n, "warmup_plain_decisions": 8}))
    del warm
    leg.free()


def sweep(args, dev):
    """The arena-count sweep (4,096 ... 1,048,576 arenas of one workload): the plain launch, the lockstep kernel and the
    lockstep kernel with the learned binning (two bins, and sixteen cost levels), each timed on the same decisions from
    the same start states; all words of the runs compared on the device, and a seeded 1% sample of the arenas replayed
    through the oracle.  One JSON line per size."""
    import torch
    import rsx
    from runner import DecisionRunner

    mix = rsx.MIX_HEADLINE if args.mix == "headline" else rsx.MIX_CONTACT_HEAVY
    L = oracle_batch()
    D = args.sweep_decisions
    for n in [int(x) for x in args.sizes.split(",")]:
        sds, idx, st = world(rsx, n, 0, args.seed, mix)
        run = DecisionRunner(dev, sds, idx, st)
        ctl_host = controls_of(rsx, args.seed * 1000, 0, D + 1, n)
        ctl = [torch.from_numpy(ctl_host[d].view(np.int32)).to(dev.device) for d in range(D + 1)]
        torch.cuda.synchronize()
        start = run.snapshot()
        t0 = time.perf_counter()
        run.train_predictor(control_seed=args.seed * 1000 + 500, decisions=max(2, 2097152 // n))
        train_s = time.perf_counter() - t0
        base = {"block": 448, "grid": run.sms, "split": 15}
        out, words = {}, {}
        for name, cfg in [("plain", {"mode": "plain", "block": 32}), ("lockstep", {"mode": "lockstep", **base}),
                          ("binned", {"mode": "binned", "threshold": 0.5, **base}),
                          ("levels", {"mode": "levels", "levels": 16, "weights": [1.0] * 6, **base})]:
            run.restore(start)
            run.step(ctl[0].data_ptr(), cfg)  # the first launch of a kernel loads it: outside the timing
            run.stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(run.stream)
            for d in range(1, D + 1):
                run.step(ctl[d].data_ptr(), cfg)
            e1.record(run.stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / D
            out[name] = {"ms_per_decision": round(ms, 3), "arena_ticks_per_s": n * 8 / (ms / 1e3)}
            words[name] = (run.snapshot(), run.res.clone())
        exact = all(torch.equal(words[k][0], words["plain"][0]) and torch.equal(words[k][1], words["plain"][1]) for k in words)
        rec = {"arenas": n, "mix": args.mix, "decisions": D, "train_s": round(train_s, 2), **out,
               "lockstep_vs_plain": out["plain"]["ms_per_decision"] / out["lockstep"]["ms_per_decision"],
               "binned_vs_plain": out["plain"]["ms_per_decision"] / out["binned"]["ms_per_decision"],
               "levels_vs_plain": out["plain"]["ms_per_decision"] / out["levels"]["ms_per_decision"],
               "bit_exact_all_arenas": bool(exact)}
        if L is not None and hasattr(L, "rsref_run_batch_ex"):
            rng = np.random.default_rng(args.seed + n)
            sample = np.sort(rng.choice(n, size=max(1, n // 100), replace=False))
            # the plain run's final words and result words of the last decision; every decision's words through the oracle
            a = torch.from_numpy(sample.astype(np.int64)).to(dev.device)[:, None]
            w = torch.arange(TICK_WORDS, device=dev.device, dtype=torch.int64)[None, :]
            pos = ((a // 32) * (32 * rsx.ARENA_WORDS) + w * 32 + (a % 32)).reshape(-1)
            got = words["plain"][0][pos].reshape(len(sample), TICK_WORDS).cpu().numpy().view(np.uint32)
            st0 = np.ascontiguousarray(st[sample])
            m = len(sample)
            res = np.zeros((D + 1, m), np.uint32)
            ev = np.zeros((D + 1, m), np.uint32)
            # every array handed to the C call by address stays referenced until the call returns
            sdsc = np.ascontiguousarray(sds)
            sidx = np.ascontiguousarray(idx[sample])
            smp = np.ascontiguousarray(sample.astype(np.uint32))
            L.rsref_run_batch_ex(st0.ctypes.data, m, sdsc.ctypes.data, sidx.ctypes.data, ctl_host.ctypes.data, n, smp.ctypes.data, D + 1, 0,
                                 res.ctypes.data, ev.ctypes.data)
            last = words["plain"][1].index_select(0, a[:, 0]).cpu().numpy().view(np.uint32)
            rec["oracle_sample"] = {"arenas": m, "decisions": D + 1,
                                    "state_mismatches": int(np.any(st0[:, :TICK_WORDS] != got, axis=1).sum()),
                                    "last_result_mismatches": int((res[-1] != last).sum())}
        print(json.dumps(rec), flush=True)
        del words, start, st
        run.free()
        del run
        torch.cuda.empty_cache()


def rollout_check(args, dev):
    """The on-device rollout of rollout.py (contact-heavy mix, the learned 16-level order retrained every 64 decisions,
    goal-ended episodes restarted on the device) with a seeded 1% sample of its arenas gathered on the device at
    decisions 1, D / 2 and D, and replayed through the oracle decision by decision (the same controls; the same restarts,
    from the host twin of the device's start-state generator), compared word for word.  One JSON line."""
    import torch
    import rsx
    import rollout
    from runner import DecisionRunner

    n, D, K = args.rollout_arenas, args.rollout_decisions, 16
    mix = rsx.MIX_CONTACT_HEAVY
    sds, idx, st = world(rsx, n, 0, args.seed, mix)
    run = DecisionRunner(dev, sds, idx, st)
    sample = np.sort(np.random.default_rng(args.seed + 4).choice(n, max(1, n // 100), replace=False))
    st0 = np.ascontiguousarray(st[sample])  # the sample's start states (the rest is on the device)
    del st
    host_pool = [rsx.decision_controls(args.seed * 1000, k, n) for k in range(K)]
    pool = [torch.from_numpy(c.view(np.int32)).to(dev.device) for c in host_pool]
    t0 = time.perf_counter()
    run.train_predictor(control_seed=args.seed * 1000 + 500, decisions=max(2, 2097152 // n))
    train_s = time.perf_counter() - t0
    a = torch.from_numpy(sample.astype(np.int64)).to(dev.device)[:, None]
    w = torch.arange(TICK_WORDS, device=dev.device, dtype=torch.int64)[None, :]
    pos = ((a // 32) * (32 * rsx.ARENA_WORDS) + w * 32 + (a % 32)).reshape(-1)
    checks = sorted({1, max(1, D // 2), D})
    got = {}

    def on_decision(d):  # after decision d and its restarts
        if d + 1 in checks:
            snap = run.snapshot()
            got[d + 1] = snap[pos].reshape(len(sample), TICK_WORDS).cpu().numpy().view(np.uint32)
            del snap

    cfg = {"mode": "levels", "block": 448, "grid": run.sms, "split": args.split, "threshold": None, "levels": 16, "weights": [1.0] * 6}
    reset_seed = args.seed * 7919
    ro = rollout.Rollout(run, pool, reset_seed=reset_seed, mix=mix, config=cfg)
    windows = ro.run_decisions(D, 64, on_decision=on_decision)
    total_ms = sum(x["ms_per_decision"] * (x["decisions"][1] - x["decisions"][0] + 1) for x in windows)
    run.free()
    # the oracle's replay of the sample
    L = oracle_batch()
    check = None
    if L is not None and hasattr(L, "rsref_run_batch_ex"):
        t1 = time.perf_counter()
        m = len(sample)
        ref = st0
        sdsc = np.ascontiguousarray(sds)
        sidx = np.ascontiguousarray(idx[sample])
        smp = np.ascontiguousarray(sample.astype(np.uint32))
        res = np.zeros((1, m), np.uint32)
        ev = np.zeros((1, m), np.uint32)
        bad, resets = {}, 0
        for d in range(D):
            ctl = host_pool[d % K]
            L.rsref_run_batch_ex(ref.ctypes.data, m, sdsc.ctypes.data, sidx.ctypes.data, ctl.ctypes.data, n, smp.ctypes.data, 1, 0,
                                 res.ctypes.data, ev.ctypes.data)
            hit = np.nonzero(res[0] & 0xFF)[0]
            if hit.size:
                resets += hit.size
                ref[hit] = rsx.make_states_at(sds, idx[sample[hit]], sample[hit], reset_seed + d, mix)
            if d + 1 in checks:
                bad[d + 1] = int(np.any(got[d + 1] != ref[:, :TICK_WORDS], axis=1).sum())
        check = {"arenas": int(m), "at_decisions": checks, "mismatches": bad, "restarts_in_sample": resets,
                 "oracle_seconds": round(time.perf_counter() - t1, 1)}
    print(json.dumps({"rollout": {"arenas": n, "decisions": D, "mix": "contact-heavy", "config": kernel_name(cfg) + " levels",
                                  "initial_train_s": round(train_s, 2), "arena_ticks_per_s": n * 8 * D / (total_ms / 1e3),
                                  "windows": [{k: (round(v, 4) if isinstance(v, float) else v) for k, v in x.items()} for x in windows]},
                      "bit_exact_vs_oracle": check}))


ZONE_NAMES = {0: "P1 car pre-tick head", 1: "P1 wheel rays", 2: "P1 wheel response", 3: "P1 car pre-tick tail", 10: "P3b pair heads",
              4: "  SAT: feature pairs (enumerate + first min)", 5: "  rays: candidates and mesh walks", 9: "    rays: the mesh walks alone", 6: "  rays: pooled leaf evaluations",
              7: "  rays: replays and hits", 8: "  rays: pool barriers (incl. the prefix sum)", 11: "P3b box-triangle SAT", 12: "P3b box BVH step", 13: "P3b box job tail", 14: "P3b sphere BVH step",
              15: "P3b sphere-triangle", 16: "P3b sphere job tail", 17: "  head: convex-plane", 18: "  head: sphere-box",
              19: "  head: box-box", 21: "  head: sphere job begin", 22: "  head: box job begin", 23: "  head: near tail",
              24: "  ray: box", 25: "  ray: sphere", 26: "  ray: plane", 27: "  ray: mesh", 28: "  ray: body setup",
              60: "copy-in (load_tick)", 61: "copy-out (store_tick)"}
for _k, _nm in enumerate(["P0", "P1", "P2", "P3a", "P3b", "P4", "P5", "P6", "P7", "P8"]):
    ZONE_NAMES[40 + _k] = "phase " + _nm
    ZONE_NAMES[50 + _k] = "barrier after " + _nm


LOCKSTEP_ZONE_NAMES = {40: "P0", 41: "P1 pre-tick head (per car)", 42: "P1 wheel rays (per car)", 43: "P1 wheel response (per car)",
                       44: "P2", 45: "P3a", 46: "P3b", 47: "P4", 48: "P5 (3 pieces)", 49: "P6", 29: "P7", 30: "P8 (2 pieces)",
                       33: "  P3b heads and walks", 34: "  P3b pooled leaf tests", 35: "  P3b additions and tails",
                       60: "copy-in (load_tick)", 61: "copy-out (store_tick)"}
for _i, _nm in zip([50, 51, 52, 53, 54, 55, 56, 57, 58, 59, 31, 32],
                   ["P0", "P1 head", "P1 rays", "P1 response", "P2", "P3a", "P3b (pool rounds)", "P4", "P5", "P6", "P7", "P8"]):
    LOCKSTEP_ZONE_NAMES[_i] = "barrier after " + _nm


def zones(args, dev):
    """Zone-timer profile of `sweep_decisions` decisions of the workload: warp cycles per phase and per barrier (and with
    --zones-all the simulator's inner markers), from the profiling builds librsx_zones.so / librsx_zones_all.so
    (`make -C rocketsim-cuda_b200 zones`; not part of librsx.so)."""
    import torch
    import rsx

    if args.zones_lockstep:
        lib = "librsx_zones_ls_all.so" if args.zones_all else "librsx_zones_ls.so"
    else:
        lib = "librsx_zones_all.so" if args.zones_all else "librsx_zones.so"
    Z = ctypes.CDLL(os.path.join(ROOT, "rocketsim-cuda_b200", lib))
    vp = ctypes.c_void_p
    if args.zones_lockstep:
        Z.rsx_zones_lockstep.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, vp, ctypes.c_uint32, ctypes.c_int, vp]
    else:
        Z.rsx_zones_decision.argtypes = [vp, ctypes.c_uint32, vp, vp, vp, vp, vp, vp]
    names = dict(LOCKSTEP_ZONE_NAMES) if args.zones_lockstep else ZONE_NAMES
    if args.zones_lockstep and args.zones_all:  # the simulator's own markers too (they inflate the pieces that hold them)
        names.update({i: "    " + nm.strip() for i, nm in ZONE_NAMES.items() if i < 29})
    n = args.arenas
    sds, idx, st = world(rsx, n, 0, args.seed, rsx.MIX_HEADLINE if args.mix == "headline" else rsx.MIX_CONTACT_HEAVY)
    dsd = dev.upload_static(sds)
    ds = dev.upload_states(st)
    didx = torch.from_numpy(idx).to(dev.device)
    res = torch.zeros(n, dtype=torch.int32, device=dev.device)
    counter = torch.zeros(1, dtype=torch.int32, device=dev.device)
    tot = np.zeros(64, np.float64)
    for d in range(args.zones_skip):  # to the states of later decisions (the bench times decisions after its warm-up)
        ctl = dev.upload_controls(rsx.decision_controls(1000, d, n))
        rsx.check(rsx.lib().rsx_sim8_multi_raw(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), res.data_ptr(), None, 32,
                                               dev.stream_ptr()), "rsx_sim8_multi_raw")
    dev.sync()
    for d in range(args.zones_skip, args.zones_skip + args.sweep_decisions):
        ctl = dev.upload_controls(rsx.decision_controls(1000, d, n))
        out = np.zeros(64, np.uint64)
        if args.zones_lockstep:
            rc = Z.rsx_zones_lockstep(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), res.data_ptr(), counter.data_ptr(), 448, args.split,
                                      out.ctypes.data)
        else:
            rc = Z.rsx_zones_decision(ds.ptr(), n, dsd.ptr(), didx.data_ptr(), ctl.data_ptr(), res.data_ptr(), counter.data_ptr(), out.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"zone run failed ({rc})")
        tot += out.astype(np.float64)
    if args.zones_lockstep:
        pieces = [40, 41, 42, 43, 44, 45, 46, 47, 48, 49, 29, 30, 33, 34, 35]  # 33-35: P3b's pieces in the pooled splits
        bars = [50, 51, 52, 53, 54, 55, 56, 57, 58, 59, 31, 32]
    else:
        pieces, bars = [40 + k for k in range(10)], [50 + k for k in range(10)]
    phases = sum(tot[i] for i in pieces)
    barriers = sum(tot[i] for i in bars)
    allc = phases + barriers
    print(f"{args.mix}, {n} arenas, {args.sweep_decisions} decisions{', lockstep split %d' % args.split if args.zones_lockstep else ''}: "
          f"warp Gcycles in phases {phases / 1e9:.2f}, at barriers {barriers / 1e9:.2f}")
    for i in sorted(names):
        if tot[i] > 0:
            print(f"  {names[i]:34s} {tot[i] / 1e9:9.3f} G  {100 * tot[i] / allc:6.2f}% of all warp cycles")
    ds.free()
    dsd.free()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
