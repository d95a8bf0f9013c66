// Test / baseline driver of the oracle: runs the reference's own CPU decision function (rscuda_step_ticks of
// crates/rocketsim-cuda/csrc/phase.cpp, linked from oracle/_ref/librsref.so) over many arenas on a std::thread pool,
// arenas split statically (the CPU-baseline plan).  Built by oracle/Makefile into oracle/_ref/librsbatch.so.
#include <stdint.h>
#include <stddef.h>
#include <thread>
#include <vector>

extern "C" int rscuda_step_ticks(void* s, const void* sd, const void* controls, uint32_t n, uint32_t* scored_tick, void* trace);

// ArenaState layout facts (cuda/sim/arena_state.cuh:201-234): 2,784 words, of which the first 2,567 cross a tick; the
// last of those is the tick's events word and the six before it are the overflow counters.
static const size_t kArenaWords = 2784, kTickWords = 2567, kStaticWords = 317895;
static const size_t kEventsWord = kTickWords - 1, kOverflowWord = kTickWords - 7, kOverflowCount = 6;
static const uint32_t kUnimplemented = 0x80000000u, kOverflow = 0x40000000u;

template <class Body>
static int pool(uint32_t n, int threads, const Body& body) {
  if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
  if (threads < 1) threads = 1;
  if ((uint32_t)threads > n) threads = (int)(n ? n : 1);
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t) {
    th.emplace_back([=] {
      uint32_t lo = (uint32_t)((uint64_t)n * t / threads), hi = (uint32_t)((uint64_t)n * (t + 1) / threads);
      body(lo, hi);
    });
  }
  for (auto& x : th) x.join();
  return threads;
}

extern "C" {
// states: n x 2784 words (in place), statics: count x 317895 words, sd_index: n bytes (null: all use statics[0]),
// controls: decisions x n x 16 words, scored: decisions x n (may be null).  Returns the number of threads used.
int rsref_run_batch(uint32_t* states, uint32_t n, const uint32_t* statics, const uint8_t* sd_index, const uint32_t* controls,
                    uint32_t decisions, int threads, uint32_t* scored) {
  return pool(n, threads, [=](uint32_t lo, uint32_t hi) {
    for (uint32_t a = lo; a < hi; ++a) {
      const uint32_t* sd = statics + (size_t)(sd_index ? sd_index[a] : 0) * kStaticWords;
      for (uint32_t d = 0; d < decisions; ++d) {
        uint32_t sc = 0;
        rscuda_step_ticks(states + (size_t)a * kArenaWords, sd, controls + ((size_t)d * n + a) * 16, 8, &sc, nullptr);
        if (scored) scored[(size_t)d * n + a] = sc;
      }
    }
  });
}

// The same, with each decision's full result word and event OR as the decision kernels write them (sim.cu:87-89 for the
// result: scored tick | UNIMPLEMENTED when a tick up to the goal was | OVERFLOW when the kept state's counters are
// non-zero; the event OR: the events word of every tick up to the scored one, from the per-tick trace).
// result, ev_or: decisions x n words each.  The controls of decision d of arena a sit at controls[(d * ctl_stride + a) * 16]
// (ctl_stride >= n, so a sample of arenas can read its rows from the whole workload's controls with an index map:
// ctl_index[a], or a itself when null).
int rsref_run_batch_ex(uint32_t* states, uint32_t n, const uint32_t* statics, const uint8_t* sd_index, const uint32_t* controls,
                       uint32_t ctl_stride, const uint32_t* ctl_index, uint32_t decisions, int threads, uint32_t* result,
                       uint32_t* ev_or) {
  return pool(n, threads, [=](uint32_t lo, uint32_t hi) {
    std::vector<uint32_t> trace(8 * kArenaWords);
    for (uint32_t a = lo; a < hi; ++a) {
      const uint32_t* sd = statics + (size_t)(sd_index ? sd_index[a] : 0) * kStaticWords;
      uint32_t* s = states + (size_t)a * kArenaWords;
      uint32_t row = ctl_index ? ctl_index[a] : a;
      for (uint32_t d = 0; d < decisions; ++d) {
        uint32_t sc = 0;
        int st = rscuda_step_ticks(s, sd, controls + ((size_t)d * ctl_stride + row) * 16, 8, &sc, trace.data());
        uint32_t upto = sc ? sc : 8, ev = 0, ovf = 0;
        for (uint32_t t = 0; t < upto; ++t) ev |= trace[(size_t)t * kArenaWords + kEventsWord];
        for (size_t k = 0; k < kOverflowCount; ++k) ovf |= s[kOverflowWord + k];
        result[(size_t)d * n + a] = sc | (st != 0 ? kUnimplemented : 0u) | (ovf ? kOverflow : 0u);
        ev_or[(size_t)d * n + a] = ev;
      }
    }
  });
}
}
