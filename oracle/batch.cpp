// Test / baseline driver of the oracle: runs the reference's own CPU decision function (rscuda_step_ticks of
// crates/rocketsim-cuda/csrc/phase.cpp, linked from oracle/_ref/librsref.so) over many arenas on a std::thread pool,
// arenas split statically (the CPU-baseline plan).  Built by oracle/Makefile into oracle/_ref/librsbatch.so.
#include <stdint.h>
#include <stddef.h>
#include <thread>
#include <vector>

extern "C" int rscuda_step_ticks(void* s, const void* sd, const void* controls, uint32_t n, uint32_t* scored_tick, void* trace);

static const size_t kArenaWords = 2784, kStaticWords = 317895;

extern "C" {
// states: n x 2784 words (in place), statics: count x 317895 words, sd_index: n bytes (null: all use statics[0]),
// controls: decisions x n x 16 words, scored: decisions x n (may be null).  Returns the number of threads used.
int rsref_run_batch(uint32_t* states, uint32_t n, const uint32_t* statics, const uint8_t* sd_index, const uint32_t* controls,
                    uint32_t decisions, int threads, uint32_t* scored) {
  if (threads <= 0) threads = (int)std::thread::hardware_concurrency();
  if (threads < 1) threads = 1;
  if ((uint32_t)threads > n) threads = (int)(n ? n : 1);
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([=] {
      uint32_t lo = (uint32_t)((uint64_t)n * t / threads), hi = (uint32_t)((uint64_t)n * (t + 1) / threads);
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
  for (auto& th : pool) th.join();
  return threads;
}
}
