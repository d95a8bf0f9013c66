// The SM-lockstep persistent decision kernel.
//
// Why: one decision runs ~10^5 dependent instructions per arena through a simulator whose machine code is about a
// megabyte (P1 and P3b alone are ~450 KB each), far beyond an SM's instruction cache.  When the warps of an SM drift
// into different phases, every warp's instruction fetches evict the others' and the SM stalls on instruction misses
// (measured on the one-thread-per-arena launch: ~26 cycles of "no instruction" stall per issued instruction, issue
// active 4% of cycles).  Here the warps of a block step their arenas phase by phase together: a __syncthreads()
// after each of the ten phases (split 1: also after each car's pre-tick inside P1; split 2: P1 of each car in three
// parts, pre-tick head / wheel rays / wheel response; split 3: also a barrier after every step of P3b's pair / leaf
// loop; split 6: split 2 with P5 as rows / iterations / integration and P8 as cars / the rest; split 7: split 6 with
// P3a one dynamic body at a time; splits 4 and 5 leave
// the barriers out between P3b (4) or P4 (5) and P8, to measure what they buy), so that at any time the block's warps
// fetch from one piece of code.  Splits 9 and 10 add the pooled contact work below; split 11 is split 10 with P3a in
// one piece again (once P3b and the rays were pooled, P3a's per-body barriers cost more than they kept together);
// split 14 is split 11 with the box-triangle SATs' feature pairs computed by the whole block; split 15 is split 14 with
// the wheel rays' mesh walks run by the whole block level by level.
//
// Work: `gridDim.x` resident blocks (normally one per SM, `blockDim.x` up to RSX_LS_MAXT threads); every warp claims
// 32 consecutive entries of `order` (arena indices; identity when null) with one atomicAdd on `counter` (zero at
// launch) whenever its previous 32 arenas have finished this launch's ticks (t_first..t_last of the decision's 8), and
// loads them at the next tick boundary.  A decision split over several launches carries each arena's progress in its
// result word (scored tick, unimplemented bit) and event word; an arena scored in an earlier launch is not stepped
// again.  The
// block leaves when no warp holds work.  Lanes past n (and order entries past n) step a copy of an arena and store nothing.
//
// Results: each arena's decision is the decide() sequence of sim/physics.cuh (controls before every tick, all 8 ticks
// stepped, the state after the first scored tick kept, event OR up to that tick), so states, result words and event
// words equal those of every other decision kernel, whatever grid, block, split or order.
//
// Compiled once per register budget (RSX_LS_MAXT threads per block, one block per SM: 448 -> 144 registers,
// 512 -> 128).
#include "kern_common.cuh"

#ifndef RSX_LS_MAXT
#define RSX_LS_MAXT 512
#endif
#define RSX_CAT2(a, b) a##b
#define RSX_CAT(a, b) RSX_CAT2(a, b)
#define K_NAME RSX_CAT(k_sim8_lockstep_t, RSX_LS_MAXT)
// Zone timers of the profiling build (RSX_ZONES; empty markers otherwise): warp cycles in each piece of the tick
// (ids 40-49 and 29-30: P0, P1 head, P1 rays, P1 response, P2, P3a, P3b, P4, P5, P6, P7, P8), at the barrier after it
// (ids 50-59 and 31-32 likewise), and inside the pooled P3b (33 heads and walks, 34 pooled tests, 35 additions).
#define LS_SYNC(id)          \
  do {                       \
    RSX_ZONE_BEGIN(zb_);     \
    __syncthreads();         \
    RSX_ZONE_END(zb_, id);   \
  } while (0)
#define L_NAME RSX_CAT(rsx_launch_sim8_lockstep_t, RSX_LS_MAXT)

namespace {
// ---- split 9: P3b with the leaf tests of every arena of the block pooled ----
// Each round, every lane whose arena has P3b work runs its pair heads up to its next mesh job and takes up to
// sim::kLeafChunk leaves of the job's BVH walk; the jobs and their (job, leaf) tests are published in shared memory
// (slots from a block-wide prefix sum); all threads of the block then run the tests, kPoolPairs at most, one test per
// thread at a time; each owner adds its hits in walk order and closes the job when its walk is done.  A heavy arena's
// leaves (a ball against a wall: up to ~30 triangles in one tick) are thus tested side by side instead of one after
// another on one lane, while the order-dependent part (the manifold updates) stays on the owner.  Jobs past the pool's
// capacity test their own leaves, as in the other splits.  Words equal every other split's: the walk / test / add
// separation is exact (sim/narrow.cuh, P3b driver).
constexpr int kPoolJobs = 128;
constexpr int kPoolPairs = 512;
// split 14: up to kDeferSat box-triangle SATs of a round that reach their 47 feature pairs have those pairs computed by
// the whole block (stage B) before their owners' threads finish them (stage C); the pairs overlay the job records, which
// no thread reads after the first stage of the tests.
constexpr int kDeferSat = 18;
struct PoolSmem {
  union {
    struct {
      sim::LeafJob job[kPoolJobs];
      const StaticData* jd[kPoolJobs];
      uint32_t pair_job[kPoolPairs];
      uint32_t pair_tri[kPoolPairs];
    };
    sim::FeatPair feat[kDeferSat][sim::kPairs];
  };
  sim::LeafHit hit[kPoolPairs];
  sim::SatFront front[kDeferSat];
  uint32_t front_pair[kDeferSat];
};
static_assert(sizeof(sim::FeatPair) * kDeferSat * sim::kPairs <=
                  sizeof(sim::LeafJob) * kPoolJobs + sizeof(void*) * kPoolJobs + sizeof(uint32_t) * 2 * kPoolPairs,
              "the feature pairs fit over the job records");
// split 10: the wheel rays' mesh leaves pooled too (sim/ray.cuh: evaluated anywhere, replayed on the owner)
constexpr int kRayJobs = 64;
constexpr int kRayPairs = 512;
constexpr int kRayJobsLane = 4;
constexpr int kRayLeavesLane = 48;
struct RayPoolSmem {
  sim::RayMeshJob job[kRayJobs];
  const StaticData* jd[kRayJobs];
  uint32_t pair_job[kRayPairs];  // job slot | mesh index << 16
  uint32_t pair_leaf[kRayPairs];
  sim::RayLeaf out[kRayPairs];
};
// split 15: the wheel rays' mesh walks pooled too.  The block walks every mesh job's BVHs level by level (front: the
// nodes of one level, each a slot | mesh << 6 | node << 10 and its path key); leaves go to a list (slot | mesh << 6 |
// leaf << 10, key), a counting sort by slot and an insertion sort by key within each slot give every job its leaves in
// the stack walk's order (sim/ray.cuh walk_expand).  Any list past its capacity sends the round to the serial walks.
constexpr int kRayFront = 256;
struct RayWalkSmem {
  sim::RayMeshJob job[kRayJobs];
  const StaticData* jd[kRayJobs];
  Box3 jbox[kRayJobs];
  uint32_t jbody[kRayJobs];
  uint32_t cnt[kRayJobs], seg[kRayJobs], fill[kRayJobs];
  uint32_t leaf_a[kRayPairs], key_a[kRayPairs];  // as found
  uint32_t leaf_b[kRayPairs], key_b[kRayPairs];  // by slot, then by key
  sim::RayLeaf out[kRayPairs];
  uint32_t front[2][kRayFront][2];
  uint32_t nfront[sim::kWalkLevels + 1], nleaf, ovf;
};
// one shared buffer for the pools (they serve different pieces of the tick) and the prefix sums
struct Pools {
  union {
    PoolSmem p3b;
    RayPoolSmem rays;
    RayWalkSmem walk;
  };
  uint32_t warp_sum[32];
  uint32_t limit;
  uint32_t deferred;  // split 14: SATs of this round whose feature pairs the block computes
};
__device__ __forceinline__ Pools& pools() {
  __shared__ Pools u;
  return u;
}

// block-wide exclusive prefix sum of v (every thread calls it); returns the exclusive sum, *total the block's sum
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t* total, Pools& sm) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
    if (lane >= (uint32_t)d) x += y;
  }
  if (lane == 31) sm.warp_sum[warp] = x;
  if (threadIdx.x == 0) {
    sm.limit = 0;
    sm.deferred = 0;
  }
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < nw ? sm.warp_sum[lane] : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, d);
      if (lane >= (uint32_t)d) w += y;
    }
    sm.warp_sum[lane] = w;
  }
  __syncthreads();
  *total = sm.warp_sum[nw - 1];
  return (warp ? sm.warp_sum[warp - 1] : 0u) + x - v;
}

// P3b of the thread's arena (have) with pooled leaf tests; every thread of the block calls it.  SplitSat (split 14): the
// box-triangle SATs that reach their feature pairs have them computed by the whole block.
template <bool SplitSat>
__device__ __noinline__ void p3b_pooled(ArenaState& s, const StaticData* D, bool have, int* un) {
  Pools& u = pools();
  PoolSmem& sm = u.p3b;
  sim::P3bLoop L;
  bool more = have;
  if (have) sim::p3b_begin(s, L);
  uint32_t tris[sim::kLeafChunk];
  for (;;) {
    int k = 0;
    bool job = false;
    RSX_ZONE_BEGIN(zo);
    if (more) {
      if (sim::p3b_open(s, *D, L) == sim::NEAR_DONE) {
        more = false;
      } else {
        job = true;
        k = sim::p3b_collect(*D, L, tris, sim::kLeafChunk);
      }
    }
    RSX_ZONE_END(zo, 33);
    // (the barrier also orders the last round's reads of the pool before this round's writes)
    RSX_ZONE_BEGIN(zb0);
    const bool any = __syncthreads_or(job);
    RSX_ZONE_END(zb0, 56);
    if (!any) break;
    uint32_t total;
    const uint32_t v = k > 0 ? ((1u << 16) | (uint32_t)k) : 0u;
    const uint32_t ex = block_scan(v, &total, u);
    const uint32_t slot = ex >> 16, off = ex & 0xFFFFu;
    // pooled jobs are a prefix in scan order (slot and off only grow), so the pool's pairs are [0, limit)
    const bool pooled = k > 0 && slot < (uint32_t)kPoolJobs && off + (uint32_t)k <= (uint32_t)kPoolPairs;
    if (pooled) {
      sim::leaf_job_of(L, sm.job[slot]);
      sm.jd[slot] = D;
      for (int i = 0; i < k; ++i) {
        sm.pair_job[off + i] = slot;
        sm.pair_tri[off + i] = tris[i];
      }
      atomicMax(&u.limit, off + (uint32_t)k);
    }
    LS_SYNC(56);
    const uint32_t npairs = u.limit;
    RSX_ZONE_BEGIN(zt);
    for (uint32_t p = threadIdx.x; p < npairs; p += blockDim.x) {
      const uint32_t j = sm.pair_job[p];
      sim::LeafHit h;
      if (!SplitSat) {
        sim::leaf_test(sm.job[j], *sm.jd[j], sm.pair_tri[p], &h);
      } else {
        sim::SatFront f;
        if (!sim::leaf_test_front(sm.job[j], *sm.jd[j], sm.pair_tri[p], &h, &f)) {
          const uint32_t d = atomicAdd(&u.deferred, 1u);
          if (d < (uint32_t)kDeferSat) {  // the block computes its feature pairs below
            sm.front[d] = f;
            sm.front_pair[d] = p;
            continue;
          }
          sim::FeatPair P[sim::kPairs];  // past the deferred capacity: this thread computes them itself
          sim::enum_pairs(f.hu, f.q, f.e, P);
          sim::leaf_test_back(f, P, &h);
        }
      }
      sm.hit[p] = h;
    }
    RSX_ZONE_END(zt, 34);
    LS_SYNC(56);
    if (SplitSat) {
      const uint32_t nd = min(u.deferred, (uint32_t)kDeferSat);
      if (nd != 0) {  // (uniform: every thread read the count after the barrier)
        RSX_ZONE_BEGIN(zf);
        for (uint32_t w = threadIdx.x; w < nd * (uint32_t)sim::kPairs; w += blockDim.x) {
          const uint32_t d = w / (uint32_t)sim::kPairs, i = w % (uint32_t)sim::kPairs;
          sm.feat[d][i] = sim::feat_pair(sm.front[d], (int)i);
        }
        RSX_ZONE_END(zf, 34);
        LS_SYNC(56);
        RSX_ZONE_BEGIN(zg);
        for (uint32_t d = threadIdx.x; d < nd; d += blockDim.x) {
          sim::LeafHit h;
          sim::leaf_test_back(sm.front[d], sm.feat[d], &h);
          sm.hit[sm.front_pair[d]] = h;
        }
        RSX_ZONE_END(zg, 34);
        LS_SYNC(56);
      }
    }
    RSX_ZONE_BEGIN(zc);
    if (pooled) {
      for (int i = 0; i < k; ++i)
        if (sm.hit[off + i].found) sim::p3b_add_hit(s, *D, L, tris[i], sm.hit[off + i]);
    } else if (k > 0) {  // past the pool's capacity: this lane tests its own leaves
      sim::LeafJob jb;
      sim::leaf_job_of(L, jb);
      for (int i = 0; i < k; ++i) {
        sim::LeafHit h;
        if (sim::leaf_test(jb, *D, tris[i], &h)) sim::p3b_add_hit(s, *D, L, tris[i], h);
      }
    }
    if (job && L.walk_done) sim::p3b_close(s, *D, L);
    RSX_ZONE_END(zc, 35);
  }
  if (have && L.unimplemented != 0) *un = 1;
}

// The wheel rays of car ci of the thread's arena (act) with the mesh leaves of the whole block pooled; every thread of
// the block calls it.  A mesh body's walk reads only the body-local rays' box, and a leaf's evaluation made with the
// starting fractions at 1 serves any later ones (sim/ray.cuh), so each lane first walks every mesh candidate of its
// packet (up to kRayJobsLane bodies, kRayLeavesLane leaves), the block evaluates all those leaves at once, and each
// owner then runs its candidates in order: mesh bodies by replaying their evaluated leaves against the fractions held
// at that point, the plane, ball and car bodies by testing them in place.  One pool round per car; results equal
// vehicle_rays'.  Lanes past the pool's capacity or their own budget run vehicle_rays' sequence.
__device__ __noinline__ void rays_pooled(ArenaState& s, const StaticData* D, bool act, int ci, sim::WheelHit hits[kWheels]) {
  Pools& u = pools();
  RayPoolSmem& sm = u.rays;
  sim::RayPacket pk;
  uint32_t cand[kHandles];
  int nk = 0;
  RSX_ZONE_BEGIN(zr0);
  if (act) {
    sim::vehicle_rays_begin(s, *D, ci, pk);
    nk = sim::grid_candidates(s, *D, &pk, cand);
  }
  uint32_t leaves[kRayLeavesLane];
  uint8_t meshes[kRayLeavesLane], jcand[kRayJobsLane], jstart[kRayJobsLane], jcount[kRayJobsLane];
  int nj = 0, nl = 0;
  bool fits = true;
  RSX_ZONE_BEGIN(zr6);
  for (int k = 0; k < nk && fits; ++k) {
    const uint32_t w = cand[k];
    const uint32_t shape = D->bodies[w].shape;
    if (shape == sim::SHAPE_BOX || shape == sim::SHAPE_SPHERE || shape == sim::SHAPE_PLANE) continue;
    if (nj == kRayJobsLane) {
      fits = false;
      break;
    }
    sim::LocalRays lr;
    sim::RayBox rb;
    sim::ray_body_setup(s, *D, w, &pk, lr, rb);
    sim::RayWalk wk;
    sim::ray_walk_seek(wk, *D, w, rb.box, 0);
    int mesh;
    uint32_t leaf;
    const int first = nl;
    while (sim::ray_walk_next(wk, *D, w, rb.box, &mesh, &leaf)) {
      if (nl == kRayLeavesLane) {
        fits = false;
        break;
      }
      leaves[nl] = leaf;
      meshes[nl] = (uint8_t)mesh;
      ++nl;
    }
    jcand[nj] = (uint8_t)k;
    jstart[nj] = (uint8_t)first;
    jcount[nj] = (uint8_t)(nl - first);
    ++nj;
  }
  RSX_ZONE_END(zr6, 9);
  if (!fits) nj = nl = 0;
  RSX_ZONE_END(zr0, 5);
  RSX_ZONE_BEGIN(zr1);
  uint32_t total;
  const uint32_t ex = block_scan(((uint32_t)nj << 16) | (uint32_t)nl, &total, u);
  const uint32_t slot = ex >> 16, off = ex & 0xFFFFu;
  // all of a lane's bodies or none; pooled lanes are a prefix in scan order
  const bool pooled = nj > 0 && slot + (uint32_t)nj <= (uint32_t)kRayJobs && off + (uint32_t)nl <= (uint32_t)kRayPairs;
  if (pooled) {
    for (int j = 0; j < nj; ++j) {  // no body has been tested yet: the packet's fractions are all still 1
      sim::LocalRays lr;
      sim::RayBox rb;
      sim::ray_body_setup(s, *D, cand[jcand[j]], &pk, lr, rb);
      sim::ray_mesh_job(lr, rb, sm.job[slot + j]);
      sm.jd[slot + j] = D;
      for (int t = 0; t < jcount[j]; ++t) {
        sm.pair_job[off + jstart[j] + t] = (slot + j) | ((uint32_t)meshes[jstart[j] + t] << 16);
        sm.pair_leaf[off + jstart[j] + t] = leaves[jstart[j] + t];
      }
    }
    atomicMax(&u.limit, off + (uint32_t)nl);
  }
  __syncthreads();
  RSX_ZONE_END(zr1, 8);
  RSX_ZONE_BEGIN(zr2);
  const uint32_t npairs = u.limit;
  for (uint32_t p = threadIdx.x; p < npairs; p += blockDim.x) {
    const uint32_t j = sm.pair_job[p] & 0xFFFFu;
    const StaticData& Dj = *sm.jd[j];
    sim::ray_leaf_eval(sm.job[j], Dj, Dj.meshes[sm.pair_job[p] >> 16], sm.pair_leaf[p], nullptr, &sm.out[p]);
  }
  RSX_ZONE_END(zr2, 6);
  RSX_ZONE_BEGIN(zr3);
  __syncthreads();
  RSX_ZONE_END(zr3, 8);
  RSX_ZONE_BEGIN(zr4);
  if (act) {
    int j = 0;
    for (int k = 0; k < nk; ++k) {
      const uint32_t w = cand[k];
      if (pooled && j < nj && jcand[j] == k) {
        sim::LocalRays lr;
        sim::RayBox rb;
        sim::ray_body_setup(s, *D, w, &pk, lr, rb);
        for (int t = 0; t < jcount[j]; ++t) {
          const int q = jstart[j] + t;
          sim::ray_leaf_replay(&lr, rb.lmax, *D, D->meshes[meshes[q]], leaves[q], sm.out[off + q]);
        }
        ++j;
      } else {
        sim::ray_body(s, *D, w, &pk);
      }
    }
    sim::wheel_packet_hits(s, *D, pk, hits);
  }
  RSX_ZONE_END(zr4, 7);
  RSX_ZONE_BEGIN(zr5);
  __syncthreads();  // the pool is read above: the next piece's writes come after every lane's reads
  RSX_ZONE_END(zr5, 8);
}

// rays_pooled with the mesh walks pooled too (split 15); every thread of the block calls it.  Each lane's mesh
// candidates (up to kRayJobsLane) become jobs in shared memory, the block walks all their BVHs level by level, sorts
// each job's leaves into the stack walk's order, evaluates them, and each owner replays its candidates in order as in
// rays_pooled.  Results equal vehicle_rays'.
__device__ __noinline__ void rays_pooled_walk(ArenaState& s, const StaticData* D, bool act, int ci, sim::WheelHit hits[kWheels]) {
  Pools& u = pools();
  RayWalkSmem& sm = u.walk;
  sim::RayPacket pk;
  uint32_t cand[kHandles];
  int nk = 0;
  RSX_ZONE_BEGIN(zr0);
  if (act) {
    sim::vehicle_rays_begin(s, *D, ci, pk);
    nk = sim::grid_candidates(s, *D, &pk, cand);
  }
  uint8_t jcand[kRayJobsLane];
  int nj = 0;
  for (int k = 0; k < nk; ++k) {
    const uint32_t shape = D->bodies[cand[k]].shape;
    if (shape == sim::SHAPE_BOX || shape == sim::SHAPE_SPHERE || shape == sim::SHAPE_PLANE) continue;
    if (nj == kRayJobsLane) {  // more mesh bodies than a lane may pool: this lane walks its own
      nj = -1;
      break;
    }
    jcand[nj++] = (uint8_t)k;
  }
  const bool mine = nj > 0;
  if (nj < 0) nj = 0;
  RSX_ZONE_END(zr0, 5);
  RSX_ZONE_BEGIN(zr1);
  uint32_t total;
  const uint32_t slot = block_scan((uint32_t)nj, &total, u);
  // pooled lanes are a prefix in scan order, so the jobs are slots [0, limit)
  const bool pooled = mine && slot + (uint32_t)nj <= (uint32_t)kRayJobs;
  if (threadIdx.x == 0) {
    for (int l = 0; l <= sim::kWalkLevels; ++l) sm.nfront[l] = 0;
    sm.nleaf = 0;
    sm.ovf = 0;
  }
  if (pooled) {
    for (int j = 0; j < nj; ++j) {  // no body has been tested yet: the packet's fractions are all still 1
      const uint32_t w = cand[jcand[j]], q = slot + (uint32_t)j;
      sim::LocalRays lr;
      sim::RayBox rb;
      sim::ray_body_setup(s, *D, w, &pk, lr, rb);
      sim::ray_mesh_job(lr, rb, sm.job[q]);
      sm.jd[q] = D;
      sm.jbox[q] = rb.box;
      sm.jbody[q] = w;
      sm.cnt[q] = 0;
      sm.fill[q] = 0;
    }
    atomicMax(&u.limit, slot + (uint32_t)nj);
  }
  __syncthreads();
  RSX_ZONE_END(zr1, 8);
  RSX_ZONE_BEGIN(zr6);
  const uint32_t J = u.limit;
  // the jobs' meshes: every mesh of the job's body whose root box meets the job's box, in mesh order by key
  for (uint32_t i = threadIdx.x; i < J * (uint32_t)kMeshes; i += blockDim.x) {
    const uint32_t q = i / (uint32_t)kMeshes;
    const int m = (int)(i % (uint32_t)kMeshes);
    const StaticData& Dj = *sm.jd[q];
    if (Dj.meshes[m].body == sm.jbody[q] && box_overlap(sm.jbox[q], Dj.meshes[m].root_box)) {
      const uint32_t f = atomicAdd(&sm.nfront[0], 1u);
      if (f < (uint32_t)kRayFront) {
        sm.front[0][f][0] = q | ((uint32_t)m << 6);
        sm.front[0][f][1] = sim::walk_root_key(m);
      } else {
        sm.ovf = 1;
      }
    }
  }
  __syncthreads();
  for (int level = 0; level < sim::kWalkLevels; ++level) {
    const uint32_t F = sm.nfront[level];
    if (F == 0 || sm.ovf) break;  // (uniform: read after the barrier, written only between barriers)
    const int cur = level & 1;
    for (uint32_t i = threadIdx.x; i < F; i += blockDim.x) {
      const uint32_t it = sm.front[cur][i][0], key = sm.front[cur][i][1];
      const uint32_t q = it & 63u, m = (it >> 6) & 15u, node = it >> 10;
      sim::walk_expand(*sm.jd[q], (int)m, node, key, level, sm.jbox[q], [&](uint32_t ch, uint32_t k2) {
        if (ch & 0x80000000u) {
          const uint32_t e = atomicAdd(&sm.nleaf, 1u);
          if (e < (uint32_t)kRayPairs) {
            sm.leaf_a[e] = q | (m << 6) | ((ch & 0x7FFFFFFFu) << 10);
            sm.key_a[e] = k2;
            atomicAdd(&sm.cnt[q], 1u);
          } else {
            sm.ovf = 1;
          }
        } else {
          const uint32_t f = atomicAdd(&sm.nfront[level + 1], 1u);
          if (f < (uint32_t)kRayFront) {
            sm.front[cur ^ 1][f][0] = q | (m << 6) | (ch << 10);
            sm.front[cur ^ 1][f][1] = k2;
          } else {
            sm.ovf = 1;
          }
        }
      });
    }
    __syncthreads();
  }
  // past a list's capacity, or a tree deeper than the keys hold: every lane walks its own this round
  const bool walked = !(sm.ovf || sm.nfront[sim::kWalkLevels] != 0);
  const uint32_t nl = walked ? sm.nleaf : 0u;
  if (walked) {
    if (threadIdx.x == 0) {
      uint32_t acc = 0;
      for (uint32_t q = 0; q < J; ++q) {
        sm.seg[q] = acc;
        acc += sm.cnt[q];
      }
    }
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < nl; e += blockDim.x) {
      const uint32_t q = sm.leaf_a[e] & 63u;
      const uint32_t at = sm.seg[q] + atomicAdd(&sm.fill[q], 1u);
      sm.leaf_b[at] = sm.leaf_a[e];
      sm.key_b[at] = sm.key_a[e];
    }
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < J; q += blockDim.x) {  // each job's leaves into key order
      const uint32_t b = sm.seg[q], n = sm.cnt[q];
      for (uint32_t i = 1; i < n; ++i) {
        const uint32_t lv = sm.leaf_b[b + i], kv = sm.key_b[b + i];
        uint32_t j = i;
        for (; j > 0 && sm.key_b[b + j - 1] > kv; --j) {
          sm.leaf_b[b + j] = sm.leaf_b[b + j - 1];
          sm.key_b[b + j] = sm.key_b[b + j - 1];
        }
        sm.leaf_b[b + j] = lv;
        sm.key_b[b + j] = kv;
      }
    }
    __syncthreads();
  }
  RSX_ZONE_END(zr6, 9);
  RSX_ZONE_BEGIN(zr2);
  for (uint32_t e = threadIdx.x; e < nl; e += blockDim.x) {
    const uint32_t v = sm.leaf_b[e], q = v & 63u;
    const StaticData& Dj = *sm.jd[q];
    sim::ray_leaf_eval(sm.job[q], Dj, Dj.meshes[(v >> 6) & 15u], v >> 10, nullptr, &sm.out[e]);
  }
  RSX_ZONE_END(zr2, 6);
  RSX_ZONE_BEGIN(zr3);
  __syncthreads();
  RSX_ZONE_END(zr3, 8);
  RSX_ZONE_BEGIN(zr4);
  if (act) {
    int j = 0;
    for (int k = 0; k < nk; ++k) {
      const uint32_t w = cand[k];
      if (walked && pooled && j < nj && jcand[j] == k) {
        sim::LocalRays lr;
        sim::RayBox rb;
        sim::ray_body_setup(s, *D, w, &pk, lr, rb);
        const uint32_t q = slot + (uint32_t)j, b = sm.seg[q], n = sm.cnt[q];
        for (uint32_t t = 0; t < n; ++t) {
          const uint32_t v = sm.leaf_b[b + t];
          sim::ray_leaf_replay(&lr, rb.lmax, *D, D->meshes[(v >> 6) & 15u], v >> 10, sm.out[b + t]);
        }
        ++j;
      } else {
        sim::ray_body(s, *D, w, &pk);
      }
    }
    sim::wheel_packet_hits(s, *D, pk, hits);
  }
  RSX_ZONE_END(zr4, 7);
  RSX_ZONE_BEGIN(zr5);
  __syncthreads();  // the pool is read above: the next piece's writes come after every lane's reads
  RSX_ZONE_END(zr5, 8);
}

}  // namespace

template <int SPLIT>
__global__ void __launch_bounds__(RSX_LS_MAXT, 1) K_NAME(uint32_t* states, const StaticData* sds, const uint8_t* sd_index,
                                                        const Controls* controls, uint32_t* result, uint32_t* ev_or,
                                                        const uint32_t* order, uint32_t* counter, uint32_t n, uint32_t t_first,
                                                        uint32_t t_last) {
  const uint32_t lane = threadIdx.x & 31u;
  ArenaState s;
  Controls c0, c1;
  const StaticData* D = sds;
  uint32_t a = 0, t = 0, scored = 0, unimpl = 0, ev = 0;
  bool live = false, have = false, ovf = false;
  for (;;) {
    // a warp without arenas claims the next 32 entries of the queue
    if (!have) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(counter, 32u);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base < n) {
        uint32_t i = base + lane;
        live = i < n;
        uint32_t j = live ? i : base;
        a = order ? order[j] : j;
        if (a >= n) {  // an order entry past n (not a permutation): step arena 0 as a copy and store nothing
          a = 0;
          live = false;
        }
        D = sds + (sd_index ? sd_index[a] : 0);
        RSX_ZONE_BEGIN(zl);
        load_tick(&s, states, a);
        RSX_ZONE_END(zl, 60);
        c0 = controls[(size_t)a * kCars];
        c1 = controls[(size_t)a * kCars + 1];
        t = t_first;
        scored = unimpl = ev = 0;
        if (t_first > 1) {  // a later launch of a split decision: the progress so far rides in the result / event words
          uint32_t r0 = result[a];
          scored = r0 & kScoredMask;
          unimpl = r0 & kUnimplemented;
          ev = ev_or ? ev_or[a] : 0u;
          if (scored) live = false;  // decided in an earlier launch (the buffer holds its goal state): store nothing
        }
        ovf = false;
        have = true;
      }
    }
    if (!__syncthreads_or(have)) break;
    // one tick, phase by phase in lockstep (every thread reaches every barrier)
    int un = 0;
    if (have) {
      s.cars[0].controls = c0;
      s.cars[1].controls = c1;
    }
    if (SPLIT >= 2) {
      {
        RSX_ZONE_BEGIN(z0);
        if (have) sim::t_p0(s, *D);
        RSX_ZONE_END(z0, 40);
      }
      LS_SYNC(50);
      if (have) {
        sim::flip_zdamp(s, *D, 0);
        sim::flip_zdamp(s, *D, 1);
      }
#pragma unroll 1
      for (int ci = 0; ci < kCars; ++ci) {
        // P1 for car ci in three barrier-separated parts: pre-tick head, wheel rays, wheel response + tail
        bool act = false;
        float rthr = 0.0f;
        uint32_t was = 0;
        RSX_ZONE_BEGIN(z1);
        if (SPLIT == 8) {  // the pre-tick head in three parts
          sim::PreTick pt;
          if (have) {
            was = s.cars[ci].on_ground;
            act = sim::car_pre_tick_wheels(s, *D, ci, pt);
          }
          __syncthreads();
          if (have && act) sim::car_pre_tick_jumps(s, *D, ci, pt);
          __syncthreads();
          if (have && act) rthr = sim::car_pre_tick_air(s, *D, ci, pt);
        } else if (have) {
          was = s.cars[ci].on_ground;
          act = sim::car_pre_tick_head(s, *D, ci, &rthr);
        }
        RSX_ZONE_END(z1, 41);
        LS_SYNC(51);
        sim::WheelHit hits[kWheels];
        {
          RSX_ZONE_BEGIN(z2);
          if (SPLIT >= 15)
            rays_pooled_walk(s, D, have && act, ci, hits);
          else if (SPLIT >= 10)
            rays_pooled(s, D, have && act, ci, hits);
          else if (have && act)
            sim::vehicle_rays(s, *D, ci, hits);
          RSX_ZONE_END(z2, 42);
        }
        LS_SYNC(52);
        {
          RSX_ZONE_BEGIN(z3);
          if (have) {
            if (act) {
              sim::vehicle_response(s, *D, ci, sim::kTickTime, s.cars[ci].handbrake_val, rthr, D->cars[ci].three_wheels != 0, hits);
              sim::car_pre_tick_tail(s, *D, ci);
            }
            if (!was && s.cars[ci].on_ground) s.events |= 1u << (EV_LANDED + ci);
          }
          RSX_ZONE_END(z3, 43);
        }
        LS_SYNC(53);
      }
#pragma unroll 1
      for (int k = 2; k < sim::kPhases; ++k) {
        // split 4: no barrier between P3b and P8 (warps without contact work run ahead to the tick's end);
        // split 5: none between P4 and P8
        const bool bar = !((SPLIT == 4 && k >= 4 && k < sim::kPhases - 1) || (SPLIT == 5 && k >= 5 && k < sim::kPhases - 1));
        // zone ids of phase k's pieces and of the barriers after them
        const int zp = k <= 7 ? 42 + k : 21 + k, zb = zp + (k <= 7 ? 10 : 2);
        (void)zp;
        (void)zb;
        if (SPLIT >= 7 && SPLIT < 11 && k == 3) {  // P3a: one dynamic body at a time (from split 11: one piece)
#pragma unroll 1
          for (uint32_t d = 0; d < (uint32_t)kDyn; ++d) {
            {
              RSX_ZONE_BEGIN(za);
              if (have) sim::t_p3a_body(s, *D, d);
              RSX_ZONE_END(za, zp);
            }
            LS_SYNC(zb);
          }
          continue;
        }
        if (SPLIT >= 6 && k == 6) {  // P5: rows, iterations, integration
          sim::Solver sv;
          RSX_ZONE_BEGIN(z5a);
          if (have) sim::t_p5_setup(s, *D, sv);
          RSX_ZONE_END(z5a, zp);
          LS_SYNC(zb);
          RSX_ZONE_BEGIN(z5b);
          if (have) sim::t_p5_iterate(sv);
          RSX_ZONE_END(z5b, zp);
          LS_SYNC(zb);
          RSX_ZONE_BEGIN(z5c);
          if (have) sim::t_p5_finish(s, *D, sv);
          RSX_ZONE_END(z5c, zp);
          LS_SYNC(zb);
          continue;
        }
        if (SPLIT >= 6 && k == 9) {  // P8: cars, then pads / ball / tick count
          RSX_ZONE_BEGIN(z8a);
          if (have) sim::t_p8_cars(s);
          RSX_ZONE_END(z8a, zp);
          LS_SYNC(zb);
          RSX_ZONE_BEGIN(z8b);
          if (have) sim::t_p8_rest(s, *D);
          RSX_ZONE_END(z8b, zp);
          LS_SYNC(zb);
          continue;
        }
        if (SPLIT == 4 || SPLIT == 5) {
          if (have && sim::run_phase(k, s, *D) != sim::PHASE_OK) un = 1;
          if (bar) __syncthreads();
          continue;
        }
        if (SPLIT >= 9 && k == 4) {  // P3b with the block's leaf tests pooled
          p3b_pooled<(SPLIT >= 14)>(s, D, have, &un);
          continue;
        }
        if (SPLIT == 3 && k == 4) {
          // P3b with a barrier after every step of the pair / leaf loop
          sim::P3bLoop L;
          bool more = have;
          if (have) sim::p3b_begin(s, L);
          while (__syncthreads_or(more))
            if (more) more = sim::t_p3b_step(s, *D, L);
          if (have && L.unimplemented != 0) un = 1;
          continue;
        }
        {
          RSX_ZONE_BEGIN(zk);
          if (have && sim::run_phase(k, s, *D) != sim::PHASE_OK) un = 1;
          RSX_ZONE_END(zk, zp);
        }
        LS_SYNC(zb);
      }
    } else if (SPLIT) {
      if (have) sim::t_p0(s, *D);
      __syncthreads();
      if (have) {
        sim::flip_zdamp(s, *D, 0);
        sim::flip_zdamp(s, *D, 1);
      }
#pragma unroll 1
      for (int ci = 0; ci < kCars; ++ci) {
        if (have) {
          uint32_t was = s.cars[ci].on_ground;
          sim::car_pre_tick(s, *D, ci);
          if (!was && s.cars[ci].on_ground) s.events |= 1u << (EV_LANDED + ci);
        }
        __syncthreads();
      }
#pragma unroll 1
      for (int k = 2; k < sim::kPhases; ++k) {
        if (have && sim::run_phase(k, s, *D) != sim::PHASE_OK) un = 1;
        __syncthreads();
      }
    } else {
#pragma unroll 1
      for (int k = 0; k < sim::kPhases; ++k) {
        if (have && sim::run_phase(k, s, *D) != sim::PHASE_OK) un = 1;
        __syncthreads();
      }
    }
    // the tick hooks of decide(): event OR, goal state, and the end of the decision
    if (have) {
      if (scored == 0) {
        if (un) unimpl = kUnimplemented;
        ev |= s.events;
        if (sim::ball_scored(s, *D)) {
          scored = t;
          if (live) store_tick(states, a, &s);
          ovf = sim::any_overflow(s);
        }
      }
      if (t == t_last) {  // the end of this launch's ticks (tick 8: of the decision)
        RSX_ZONE_BEGIN(zs);
        if (scored == 0) {
          if (live) store_tick(states, a, &s);
          ovf = sim::any_overflow(s);
        }
        RSX_ZONE_END(zs, 61);
        if (live) {
          if (ev_or) ev_or[a] = ev;
          result[a] = scored | unimpl | (ovf ? kOverflow : 0u);
        }
        have = false;
      }
      ++t;
    }
  }
}

cudaError_t L_NAME(uint32_t* states, const void* sds, const uint8_t* sd_index, const void* controls, uint32_t* result, uint32_t* ev_or,
                   const uint32_t* order, uint32_t* counter, uint32_t n, uint32_t grid, uint32_t block, int split, uint32_t t_first,
                   uint32_t t_last, cudaStream_t s) {
  const StaticData* D = (const StaticData*)sds;
  const Controls* C = (const Controls*)controls;
#define RSX_LS_LAUNCH(k) K_NAME<k><<<grid, block, 0, s>>>(states, D, sd_index, C, result, ev_or, order, counter, n, t_first, t_last)
  switch (split) {
    case 15: RSX_LS_LAUNCH(15); break;
    case 14: RSX_LS_LAUNCH(14); break;
    case 11: RSX_LS_LAUNCH(11); break;
    case 10: RSX_LS_LAUNCH(10); break;
    case 9: RSX_LS_LAUNCH(9); break;
    case 8: RSX_LS_LAUNCH(8); break;
    case 7: RSX_LS_LAUNCH(7); break;
    case 6: RSX_LS_LAUNCH(6); break;
    case 5: RSX_LS_LAUNCH(5); break;
    case 4: RSX_LS_LAUNCH(4); break;
    case 3: RSX_LS_LAUNCH(3); break;
    case 2: RSX_LS_LAUNCH(2); break;
    case 1: RSX_LS_LAUNCH(1); break;
    default: RSX_LS_LAUNCH(0); break;
  }
#undef RSX_LS_LAUNCH
  return cudaGetLastError();
}

#ifdef RSX_ZONES
// Zone-timer profiling build (not part of librsx.so): one decision of this kernel with zone sums over all warps.
__device__ unsigned long long rsx_zone_acc[148 * 16][64];
extern "C" int rsx_zones_lockstep(uint32_t* d_states, uint32_t n, const void* d_statics, const uint8_t* d_sd_index, const void* d_controls,
                                  uint32_t* d_result, uint32_t* d_counter, uint32_t block, int split, unsigned long long* zone_cycles) {
  static unsigned long long acc[148 * 16][64];
  memset(acc, 0, sizeof(acc));
  if (cudaMemcpyToSymbol(rsx_zone_acc, acc, sizeof(acc)) != cudaSuccess) return -2;
  if (cudaMemset(d_counter, 0, 4) != cudaSuccess) return -2;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  if (L_NAME(d_states, d_statics, d_sd_index, d_controls, d_result, nullptr, nullptr, d_counter, n, sms < 148 ? sms : 148, block, split, 1,
             kTicksPerDecision, 0) != cudaSuccess)
    return -2;
  if (cudaDeviceSynchronize() != cudaSuccess) return -2;
  if (cudaMemcpyFromSymbol(acc, rsx_zone_acc, sizeof(acc)) != cudaSuccess) return -2;
  for (int z = 0; z < 64; ++z) {
    zone_cycles[z] = 0;
    for (int w = 0; w < 148 * 16; ++w) zone_cycles[z] += acc[w][z];
  }
  return 0;
}
#endif
