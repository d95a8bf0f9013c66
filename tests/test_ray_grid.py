"""The wheel rays' candidate walk (sim/ray.cuh grid_candidates) finds a cell's dynamic entries by a binary search of the
ray grid's dynamic list, which is exact because the list stays sorted by cell.  Host build (g++, the simulator's float
policy) over 3,072 arenas x 80 ticks of contact-rich play: the list is sorted after every tick's P3a, and for both cars
at every tick the candidates equal those of a scan of the whole list (the reference's form), in the same order."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "rocketsim-cuda_b200", "csrc")

PROGRAM = r"""
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
// grid_candidates with the whole dynamic list scanned for each cell
static int candidates_by_scan(const ArenaState& S, const StaticData& D, const sim::RayPacket* pk, uint32_t cand[kHandles]) {
  Box3 rbx;
  rbx.lo = vmin(pk->from[0], pk->to[0]);
  rbx.hi = vmax(pk->from[0], pk->to[0]);
  for (int i = 1; i < 4; ++i) {
    rbx.lo = vmin(rbx.lo, vmin(pk->from[i], pk->to[i]));
    rbx.hi = vmax(rbx.hi, vmax(pk->from[i], pk->to[i]));
  }
  uint32_t cells[4];
  int nc = 0;
  for (int r = 0; r < 4; ++r) {
    uint32_t i3[3];
    sim::cell_indices(D, pk->from[r], i3);
    uint32_t c = sim::cell_of(D, i3);
    bool seen = false;
    for (int k = 0; k < nc; ++k) seen = seen || cells[k] == c;
    if (!seen) cells[nc++] = c;
  }
  uint32_t seen = 0;
  int nk = 0;
  for (int ci = 0; ci < nc; ++ci) {
    const CellRange& cr = D.cells[cells[ci]];
    for (uint32_t e = 0; e < cr.count; ++e) {
      uint32_t h = D.cell_handles[cr.first + e];
      if (seen & (1u << h)) continue;
      seen |= 1u << h;
      if (box_overlap(rbx, sim::proxy_box(S, D, h)) && sim::ray_accepts(D, h, pk)) cand[nk++] = D.proxies[h].body;
    }
    for (uint32_t e = 0; e < S.n_dyn_cells; ++e) {
      if (S.dyn_cells[e].cell != cells[ci]) continue;
      uint32_t h = S.dyn_cells[e].handle;
      if (seen & (1u << h)) continue;
      seen |= 1u << h;
      if (box_overlap(rbx, sim::proxy_box(S, D, h)) && sim::ray_accepts(D, h, pk)) cand[nk++] = D.proxies[h].body;
    }
  }
  return nk;
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
  long checks = 0, unsorted = 0, differ = 0, with_dyn = 0;
  ArenaState* T = new ArenaState;
  for (int a = 0; a < n; ++a) {
    ArenaState& S = *reinterpret_cast<ArenaState*>(&st[(size_t)a * kArenaWords]);
    const StaticData& D = *reinterpret_cast<const StaticData*>(&sds[(size_t)idx[a] * kStaticWords]);
    for (int t = 0; t < decisions * 8; ++t) {
      for (int c = 0; c < 2; ++c) {
        Controls& k = S.cars[c].controls;
        k.throttle = (float)(((a + t + c) % 3) - 1);
        k.steer = (float)(((a * 7 + t / 3 + c) % 3) - 1);
        k.jump = ((a + t / 5 + c) % 4) == 0;
        k.boost = ((a + t / 2) % 3) == 0;
      }
      sim::t_p0(S, D);
      std::memcpy(T, &S, sizeof S);
      for (int ci = 0; ci < 2; ++ci) {  // the packets P1 casts (on a copy: the begin step records the hard points)
        sim::RayPacket pk;
        sim::vehicle_rays_begin(*T, D, ci, pk);
        uint32_t c0[kHandles], c1[kHandles];
        int n0 = sim::grid_candidates(*T, D, &pk, c0), n1 = candidates_by_scan(*T, D, &pk, c1);
        ++checks;
        if (n0 != n1 || std::memcmp(c0, c1, sizeof(uint32_t) * (size_t)n0) != 0) ++differ;
        for (int k = 0; k < n1; ++k) with_dyn += D.bodies[c1[k]].shape == sim::SHAPE_SPHERE || D.bodies[c1[k]].shape == sim::SHAPE_BOX;
      }
      sim::t_p1(S, D); sim::t_p2(S, D); sim::t_p3a(S, D);
      for (uint32_t e = 1; e < S.n_dyn_cells; ++e) unsorted += S.dyn_cells[e - 1].cell > S.dyn_cells[e].cell;
      sim::t_p3b(S, D); sim::t_p4(S, D); sim::t_p5(S, D); sim::t_p6(S, D); sim::t_p7(S, D); sim::t_p8(S, D);
    }
  }
  std::printf("packets %ld dynamic-candidates %ld unsorted %ld differ %ld\n", checks, with_dyn, unsorted, differ);
  return unsorted != 0 || differ != 0;
}
"""


def test_dynamic_cell_search_equals_scan(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    libdir = os.path.join(ROOT, "rocketsim-cuda_b200")
    if not os.path.exists(os.path.join(libdir, "librsx.so")):
        pytest.skip("librsx.so is not built")
    src = tmp_path / "ray_grid.cpp"
    exe = tmp_path / "ray_grid"
    src.write_text(PROGRAM)
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", CSRC, str(src), "-L", libdir, "-lrsx", f"-Wl,-rpath,{libdir}",
           "-o", str(exe)]
    cuda_lib = "/usr/local/cuda/lib64"
    if os.path.isdir(cuda_lib):
        cmd[-2:-2] = ["-L", cuda_lib, f"-Wl,-rpath,{cuda_lib}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    words = out.stdout.split()
    assert int(words[words.index("dynamic-candidates") + 1]) > 100, out.stdout  # the dynamic entries were exercised


P3A_PROGRAM = r"""
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
// a body's move to another cell as the list rule states it: the old block's entries out (a pass over the whole list,
// freed slots zeroed), then the new block's in
static void move_plain(ArenaState& S, const StaticData& D, uint32_t h, const uint32_t old_idx[3], const uint32_t new_idx[3]) {
  uint32_t lo[3], hi[3];
  sim::dyn_block_range(D, old_idx, lo, hi);
  const uint32_t ny = D.grid_n[1], nz = D.grid_n[2];
  uint32_t removed = 0, n = S.n_dyn_cells < (uint32_t)kMaxDynCells ? S.n_dyn_cells : (uint32_t)kMaxDynCells, w = 0;
  for (uint32_t r = 0; r < n; ++r) {
    DynCell e = S.dyn_cells[r];
    if (e.handle == h) {
      uint32_t i = e.cell / (ny * nz), j = (e.cell / nz) % ny, k = e.cell % nz;
      if (i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] && k >= lo[2] && k <= hi[2]) {
        uint32_t bit = 1u << ((i - lo[0]) * 9 + (j - lo[1]) * 3 + (k - lo[2]));
        if (!(removed & bit)) { removed |= bit; continue; }
      }
    }
    if (w != r) S.dyn_cells[w] = e;
    ++w;
  }
  for (uint32_t r = w; r < n; ++r) S.dyn_cells[r] = DynCell{0, 0};
  S.n_dyn_cells = w;
  sim::dyn_cells_block(S, D, true, h, new_idx);
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
  long moves = 0, differ = 0;
  ArenaState* T = new ArenaState;
  for (int a = 0; a < n; ++a) {
    ArenaState& S = *reinterpret_cast<ArenaState*>(&st[(size_t)a * kArenaWords]);
    const StaticData& D = *reinterpret_cast<const StaticData*>(&sds[(size_t)idx[a] * kStaticWords]);
    for (int t = 0; t < decisions * 8; ++t) {
      for (int c = 0; c < 2; ++c) {
        Controls& k = S.cars[c].controls;
        k.throttle = 1.0f;
        k.steer = (float)(((a * 7 + t / 9 + c) % 3) - 1);
        k.boost = ((a + t / 2 + c) % 2) == 0;
        k.jump = ((a + t / 7 + c) % 6) == 0;
      }
      sim::t_p0(S, D); sim::t_p1(S, D); sim::t_p2(S, D);
      // every body's move this tick, replayed on a copy by the plain rule from the same list
      std::memcpy(T, &S, sizeof S);
      sim::t_p3a(S, D);
      for (uint32_t d = 0; d < (uint32_t)kDyn; ++d) {
        if (S.dyn_proxy[d].cell == T->dyn_proxy[d].cell) continue;
        ++moves;
        move_plain(*T, D, D.dyn_handle[d], T->dyn_proxy[d].idx, S.dyn_proxy[d].idx);
        for (int x = 0; x < 3; ++x) T->dyn_proxy[d].idx[x] = S.dyn_proxy[d].idx[x];
        T->dyn_proxy[d].cell = S.dyn_proxy[d].cell;
      }
      if (std::memcmp(T->dyn_cells, S.dyn_cells, sizeof S.dyn_cells) != 0 || T->n_dyn_cells != S.n_dyn_cells ||
          T->overflow[OVF_DYN_CELLS] != S.overflow[OVF_DYN_CELLS]) ++differ;
      sim::t_p3b(S, D); sim::t_p4(S, D); sim::t_p5(S, D); sim::t_p6(S, D); sim::t_p7(S, D); sim::t_p8(S, D);
    }
  }
  std::printf("moves %ld differ %ld\n", moves, differ);
  return differ != 0;
}
"""


def test_cell_moves_equal_plain_list_rule(tmp_path):
    """P3a's update of the dynamic-cell list when a body changes cell (the removal started at the old block's first
    cell, the freed slots zeroed once after the insertion) against the plain rule (a pass over the whole list, freed
    slots zeroed, then the insertion): the same list words, count and overflow count, on 3,072 arenas x 80 ticks of
    driving."""
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    libdir = os.path.join(ROOT, "rocketsim-cuda_b200")
    if not os.path.exists(os.path.join(libdir, "librsx.so")):
        pytest.skip("librsx.so is not built")
    src = tmp_path / "cell_moves.cpp"
    exe = tmp_path / "cell_moves"
    src.write_text(P3A_PROGRAM)
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", CSRC, str(src), "-L", libdir, "-lrsx", f"-Wl,-rpath,{libdir}",
           "-o", str(exe)]
    cuda_lib = "/usr/local/cuda/lib64"
    if os.path.isdir(cuda_lib):
        cmd[-2:-2] = ["-L", cuda_lib, f"-Wl,-rpath,{cuda_lib}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    words = out.stdout.split()
    assert int(words[words.index("moves") + 1]) > 1000, out.stdout
