"""The box-triangle SAT in stages (sim/sat.cuh: sat_front, feat_pair, sat_back), as the lockstep kernel's split 14 runs
it with each feature pair on its own thread, against the one-call box_triangle_sat and enum_pairs of the same source:
host build (g++, -ffp-contract=off, the simulator's float policy), bit for bit, on random boxes and triangles and on
the cases with ties (triangles on a box face, degenerate triangles)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "rocketsim-cuda_b200", "csrc")

PROGRAM = r"""
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdint>
#include "sim/sat.cuh"
using namespace rsx;
using namespace rsx::sim;
static uint64_t st = 0x9E3779B97F4A7C15ull;
static float rnd(float lo, float hi) {  // xorshift64*, uniform in [lo, hi)
  st ^= st >> 12; st ^= st << 25; st ^= st >> 27;
  uint32_t r = (uint32_t)((st * 0x2545F4914F6CDD1Dull) >> 40);
  return lo + (hi - lo) * (float)r / 16777216.0f;
}
static float snap(float x, int mode) { return mode ? (float)(int)(x * 4.0f) / 4.0f : x; }  // grid points: ties
int main() {
  long cases = 0, pairs_cases = 0, hits = 0, bad = 0;
  for (int it = 0; it < 200000; ++it) {
    const int mode = it % 4;  // 0: random, 1: on a quarter grid, 2: a triangle on a box face, 3: degenerate triangles
    V3 hu = v3(snap(rnd(0.25f, 2.0f), mode), snap(rnd(0.25f, 2.0f), mode), snap(rnd(0.25f, 2.0f), mode));
    float margin = rnd(0.0f, 0.1f), maxd = rnd(0.01f, 0.6f);
    V3 q[3];
    for (int k = 0; k < 3; ++k) q[k] = v3(snap(rnd(-2.5f, 2.5f), mode), snap(rnd(-2.5f, 2.5f), mode), snap(rnd(-2.5f, 2.5f), mode));
    if (mode == 2) {  // all three vertices on the +z face plane (or just off it)
      float z = hu.z + (it % 8 == 2 ? 0.0f : rnd(-0.05f, 0.05f));
      for (int k = 0; k < 3; ++k) q[k].z = z;
    }
    if (mode == 3) q[2] = q[0] + (q[1] - q[0]) * 0.5f;  // collinear
    Q4 qr = {rnd(-1, 1), rnd(-1, 1), rnd(-1, 1), rnd(-1, 1)};
    float nq = std::sqrt(qr.x * qr.x + qr.y * qr.y + qr.z * qr.z + qr.w * qr.w);
    qr = {qr.x / nq, qr.y / nq, qr.z / nq, qr.w / nq};
    Aff xf = {it % 3 ? m3_from_quat(qr) : m3_identity(), v3(rnd(-10, 10), rnd(-10, 10), rnd(-1, 5))};
    SatHit a = {}, b = {};
    bool ra = box_triangle_sat(xf, hu, margin, q, maxd, &a);
    SatFront f;
    int r = sat_front(xf, hu, margin, q, maxd, &b, &f);
    bool rb;
    if (r == SAT_PAIRS) {
      ++pairs_cases;
      FeatPair P[kPairs], R[kPairs];
      enum_pairs(f.hu, f.q, f.e, R);
      for (int i = 0; i < kPairs; ++i) P[i] = feat_pair(f, i);
      if (std::memcmp(P, R, sizeof P) != 0) { if (bad < 5) std::printf("pairs differ at case %d\n", it); ++bad; }
      rb = sat_back(f, P, &b);
    } else {
      rb = r == SAT_HIT;
    }
    ++cases;
    hits += ra;
    if (ra != rb || (ra && std::memcmp(&a, &b, sizeof a) != 0)) { if (bad < 5) std::printf("result differs at case %d\n", it); ++bad; }
  }
  std::printf("cases %ld feature-pair cases %ld hits %ld mismatches %ld\n", cases, pairs_cases, hits, bad);
  return bad != 0;
}
"""


def test_sat_stages_equal_one_call(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "sat_stages.cpp"
    exe = tmp_path / "sat_stages"
    src.write_text(PROGRAM)
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", CSRC, str(src), "-o", str(exe)], check=True,
                   capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    words = out.stdout.split()
    n_pairs, n_hits = int(words[words.index("feature-pair") + 2]), int(words[words.index("hits") + 1])
    assert n_pairs > 10000 and n_hits > 10000, out.stdout  # both the feature-pair path and hits are exercised


P3B_PROGRAM = r"""
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <vector>
#include "state.cuh"
#include "sim/physics.cuh"
using namespace rsx;
extern "C" int rsx_build_static(uint32_t* words, uint64_t seed, int p0, int p1);
extern "C" int rsx_make_states_multi(const uint32_t* sds, uint32_t count, const uint8_t* idx, uint32_t* out, uint32_t n,
                                     uint64_t seed, const float* mix);
// P3b as the lockstep kernel's split 14 runs it for one arena: rounds of open / collect, the leaves' tests in stages
// (a SAT that reaches its feature pairs finishes from feat_pair, or from enum_pairs past the deferred capacity), the
// hits added in walk order
static uint32_t p3b_staged(ArenaState& S, const StaticData& D, long* deferred) {
  sim::P3bLoop L;
  sim::p3b_begin(S, L);
  uint32_t tris[sim::kLeafChunk];
  while (sim::p3b_open(S, D, L) != sim::NEAR_DONE) {
    int k = sim::p3b_collect(D, L, tris, sim::kLeafChunk);
    sim::LeafJob jb;
    sim::leaf_job_of(L, jb);
    sim::LeafHit h[sim::kLeafChunk];
    for (int i = 0; i < k; ++i) {
      sim::SatFront f;
      if (sim::leaf_test_front(jb, D, tris[i], &h[i], &f)) continue;
      ++*deferred;
      sim::FeatPair P[sim::kPairs];
      if (i % 2 == 0)
        for (int t = 0; t < sim::kPairs; ++t) P[t] = sim::feat_pair(f, t);
      else
        sim::enum_pairs(f.hu, f.q, f.e, P);
      sim::leaf_test_back(f, P, &h[i]);
    }
    for (int i = 0; i < k; ++i)
      if (h[i].found) sim::p3b_add_hit(S, D, L, tris[i], h[i]);
    if (L.walk_done) sim::p3b_close(S, D, L);
  }
  return L.unimplemented;
}
int main() {
  const int n = 3072, decisions = 10;
  std::vector<uint32_t> sds((size_t)49 * kStaticWords);
  for (int p = 0; p < 7; ++p)
    for (int q = 0; q < 7; ++q) rsx_build_static(&sds[(size_t)(p * 7 + q) * kStaticWords], 7, p, q);
  std::vector<uint8_t> idx(n);
  for (int a = 0; a < n; ++a) idx[a] = (uint8_t)((a * 37u + 11u) % 49u);
  std::vector<uint32_t> st((size_t)n * kArenaWords);
  const float mix[5] = {0.1f, 0.3f, 0.2f, 0.3f, 0.1f};
  rsx_make_states_multi(sds.data(), 49, idx.data(), st.data(), n, 5, mix);
  long ticks = 0, bad = 0, deferred = 0;
  ArenaState* T = new ArenaState;
  for (int a = 0; a < n; ++a) {
    ArenaState& S = *reinterpret_cast<ArenaState*>(&st[(size_t)a * kArenaWords]);
    const StaticData& D = *reinterpret_cast<const StaticData*>(&sds[(size_t)idx[a] * kStaticWords]);
    for (int t = 0; t < decisions * 8; ++t) {
      for (int c = 0; c < 2; ++c) {  // controls that change every tick: throttle, steer and jumps cycling
        Controls& k = S.cars[c].controls;
        k.throttle = (float)(((a + t + c) % 3) - 1);
        k.steer = (float)(((a * 7 + t / 3 + c) % 3) - 1);
        k.jump = ((a + t / 5 + c) % 4) == 0;
        k.boost = ((a + t / 2) % 3) == 0;
      }
      sim::t_p0(S, D); sim::t_p1(S, D); sim::t_p2(S, D); sim::t_p3a(S, D);
      std::memcpy(T, &S, sizeof S);
      uint32_t u0 = sim::t_p3b(S, D);
      uint32_t u1 = p3b_staged(*T, D, &deferred);
      ++ticks;
      if (u0 != u1 || std::memcmp(T, &S, sizeof S) != 0) ++bad;
      sim::t_p4(S, D); sim::t_p5(S, D); sim::t_p6(S, D); sim::t_p7(S, D); sim::t_p8(S, D);
    }
  }
  std::printf("arena-ticks %ld deferred %ld mismatches %ld\n", ticks, deferred, bad);
  return bad != 0;
}
"""


def test_staged_p3b_equals_phase3b(tmp_path):
    """P3b with split 14's staged leaf tests, emulated arena by arena on the host, against the simulator's phase3b:
    the whole arena state after P3b, word for word, on 3,072 arenas x 80 ticks of contact-rich play."""
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    libdir = os.path.join(ROOT, "rocketsim-cuda_b200")
    if not os.path.exists(os.path.join(libdir, "librsx.so")):
        pytest.skip("librsx.so is not built")
    src = tmp_path / "p3b_staged.cpp"
    exe = tmp_path / "p3b_staged"
    src.write_text(P3B_PROGRAM)
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", CSRC, str(src), "-L", libdir, "-lrsx", f"-Wl,-rpath,{libdir}",
           "-o", str(exe)]
    cuda_lib = "/usr/local/cuda/lib64"
    if os.path.isdir(cuda_lib):
        cmd[-2:-2] = ["-L", cuda_lib, f"-Wl,-rpath,{cuda_lib}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    words = out.stdout.split()
    assert int(words[words.index("deferred") + 1]) > 1000, out.stdout  # the staged SATs ran
