"""The wheel rays' mesh walk level by level (sim/ray.cuh walk_expand and path keys), as the lockstep kernel's split 15
runs it over the whole block, against the stack walk ray_walk_next: for random boxes against every mesh body of all 49
car pairings' worlds, the leaves of the level-by-level walk sorted by key equal the stack walk's leaves in its order
(host build, bit for bit)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "rocketsim-cuda_b200", "csrc")

PROGRAM = r"""
#include <algorithm>
#include <cstdio>
#include <cstdint>
#include <vector>
#include "state.cuh"
#include "sim/physics.cuh"
using namespace rsx;
extern "C" int rsx_build_static(uint32_t* words, uint64_t seed, int p0, int p1);
static uint64_t st = 0x2545F4914F6CDD1Dull;
static float rnd(float lo, float hi) {
  st ^= st >> 12; st ^= st << 25; st ^= st >> 27;
  return lo + (hi - lo) * (float)((uint32_t)((st * 0x2545F4914F6CDD1Dull) >> 40)) / 16777216.0f;
}
int main() {
  std::vector<uint32_t> w(kStaticWords);
  long boxes = 0, leaves = 0, bad = 0, deep = 0;
  for (int p = 0; p < 7; ++p)
    for (int q = 0; q < 7; ++q) {
      rsx_build_static(w.data(), 7, p, q);
      const StaticData& D = *reinterpret_cast<const StaticData*>(w.data());
      for (uint32_t body = 0; body < (uint32_t)kBodies; ++body) {
        if (D.bodies[body].shape != sim::SHAPE_MESH) continue;
        Box3 all = {v3(1e30f, 1e30f, 1e30f), v3(-1e30f, -1e30f, -1e30f)};
        for (int m = 0; m < kMeshes; ++m)
          if (D.meshes[m].body == body) { all.lo = vmin(all.lo, D.meshes[m].root_box.lo); all.hi = vmax(all.hi, D.meshes[m].root_box.hi); }
        if (all.lo.x > all.hi.x) continue;
        for (int it = 0; it < 400; ++it) {
          V3 c = v3(rnd(all.lo.x, all.hi.x), rnd(all.lo.y, all.hi.y), rnd(all.lo.z, all.hi.z));
          float e = it % 4 == 0 ? rnd(100.0f, 2000.0f) : rnd(1.0f, 150.0f);
          Box3 box = {c - v3(e, rnd(1.0f, e), rnd(1.0f, e)), c + v3(rnd(1.0f, e), e, rnd(1.0f, e))};
          ++boxes;
          std::vector<uint64_t> serial;  // mesh << 32 | leaf, in the stack walk's order
          sim::RayWalk wk;
          sim::ray_walk_seek(wk, D, body, box, 0);
          int mesh;
          uint32_t leaf;
          while (sim::ray_walk_next(wk, D, body, box, &mesh, &leaf)) serial.push_back((uint64_t)mesh << 32 | leaf);
          struct Item { int m; uint32_t node, key; };
          std::vector<Item> front, next;
          std::vector<std::pair<uint32_t, uint64_t>> found;  // key, mesh << 32 | leaf
          for (int m = 0; m < kMeshes; ++m)
            if (D.meshes[m].body == body && box_overlap(box, D.meshes[m].root_box)) front.push_back({m, 0u, sim::walk_root_key(m)});
          for (int level = 0; !front.empty(); ++level) {
            if (level >= sim::kWalkLevels) { ++deep; break; }
            next.clear();
            for (const Item& x : front)
              sim::walk_expand(D, x.m, x.node, x.key, level, box, [&](uint32_t ch, uint32_t k2) {
                if (ch & 0x80000000u) found.push_back({k2, (uint64_t)x.m << 32 | (ch & 0x7FFFFFFFu)});
                else next.push_back({x.m, ch, k2});
              });
            std::swap(front, next);
          }
          std::sort(found.begin(), found.end());
          leaves += (long)serial.size();
          bool same = found.size() == serial.size();
          for (size_t i = 0; same && i < found.size(); ++i) same = found[i].second == serial[i];
          bad += !same;
        }
      }
    }
  std::printf("boxes %ld leaves %ld too-deep %ld mismatches %ld\n", boxes, leaves, deep, bad);
  return bad != 0 || deep != 0;
}
"""


def test_level_walk_sorted_by_key_equals_stack_walk(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    libdir = os.path.join(ROOT, "rocketsim-cuda_b200")
    if not os.path.exists(os.path.join(libdir, "librsx.so")):
        pytest.skip("librsx.so is not built")
    src = tmp_path / "walk_levels.cpp"
    exe = tmp_path / "walk_levels"
    src.write_text(PROGRAM)
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
    assert int(words[words.index("leaves") + 1]) > 10000, out.stdout
