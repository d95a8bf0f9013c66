// The whole tick: phases P0..P8 in V3's order, the goal test and the 8-tick decision (reference:
// cuda/sim/arena_step.cuh:31-105 and phase.cuh:32-46).  Host and device compile the same source.
#pragma once
#include "game.cuh"
#include "car.cuh"
#include "broad.cuh"
#include "narrow.cuh"
#include "solver.cuh"

namespace rsx {
namespace sim {

enum : int { PHASE_OK = 0, PHASE_UNIMPLEMENTED = -1, PHASE_BAD_INDEX = -2 };
constexpr int kPhases = 10;

// each phase is one out-of-line function on the device (one copy shared by every kernel that ticks)
RSX_HD RSX_NOINL inline void t_p0(ArenaState& S, const StaticData& D) { phase0(S, D); }
RSX_HD RSX_NOINL inline void t_p1(ArenaState& S, const StaticData& D) { phase1(S, D); }
RSX_HD RSX_NOINL inline void t_p2(ArenaState& S, const StaticData& D) { phase2(S, D); }
RSX_HD RSX_NOINL inline void t_p3a(ArenaState& S, const StaticData& D) { phase3a(S, D); }
RSX_HD RSX_NOINL inline void t_p3a_body(ArenaState& S, const StaticData& D, uint32_t d) { phase3a_body(S, D, d); }
RSX_HD RSX_NOINL inline uint32_t t_p3b(ArenaState& S, const StaticData& D) { return phase3b(S, D); }
RSX_HD RSX_NOINL inline bool t_p3b_step(ArenaState& S, const StaticData& D, P3bLoop& L) { return p3b_step(S, D, L); }
RSX_HD RSX_NOINL inline void t_p4(ArenaState& S, const StaticData& D) { phase4(S, D); }
RSX_HD RSX_NOINL inline void t_p5(ArenaState& S, const StaticData& D) { phase5(S, D); }
RSX_HD RSX_NOINL inline void t_p5_setup(ArenaState& S, const StaticData& D, Solver& sv) { phase5_setup(S, D, sv); }
RSX_HD RSX_NOINL inline void t_p5_iterate(Solver& sv) { phase5_iterate(sv); }
RSX_HD RSX_NOINL inline void t_p5_finish(ArenaState& S, const StaticData& D, Solver& sv) { phase5_finish(S, D, sv); }
RSX_HD RSX_NOINL inline void t_p8_cars(ArenaState& S) { phase8_cars(S); }
RSX_HD RSX_NOINL inline void t_p8_rest(ArenaState& S, const StaticData& D) { phase8_rest(S, D); }
RSX_HD RSX_NOINL inline void t_p6(ArenaState& S, const StaticData& D) { phase6(S, D); }
RSX_HD RSX_NOINL inline void t_p7(ArenaState& S, const StaticData& D) { phase7(S, D); }
RSX_HD RSX_NOINL inline void t_p8(ArenaState& S, const StaticData& D) { phase8(S, D); }

RSX_HD inline int run_phase(int k, ArenaState& S, const StaticData& D) {
  switch (k) {
    case 0: t_p0(S, D); return PHASE_OK;
    case 1: t_p1(S, D); return PHASE_OK;
    case 2: t_p2(S, D); return PHASE_OK;
    case 3: t_p3a(S, D); return PHASE_OK;
    case 4: return t_p3b(S, D) == 0 ? PHASE_OK : PHASE_UNIMPLEMENTED;
    case 5: t_p4(S, D); return PHASE_OK;
    case 6: t_p5(S, D); return PHASE_OK;
    case 7: t_p6(S, D); return PHASE_OK;
    case 8: t_p7(S, D); return PHASE_OK;
    case 9: t_p8(S, D); return PHASE_OK;
    default: return PHASE_BAD_INDEX;
  }
}

RSX_HD inline int step_tick(ArenaState& S, const StaticData& D) {
  t_p0(S, D);
  t_p1(S, D);
  t_p2(S, D);
  t_p3a(S, D);
  uint32_t un = t_p3b(S, D);
  t_p4(S, D);
  t_p5(S, D);
  t_p6(S, D);
  t_p7(S, D);
  t_p8(S, D);
  return un == 0 ? PHASE_OK : PHASE_UNIMPLEMENTED;
}

RSX_F bool ball_scored(const ArenaState& S, const StaticData& D) {
  V3 p = S.bodies[0].xf.t * kBTtoUU;
  return fabs_(p.y) > fadd(D.goal_y, D.mut[M_BALL_RADIUS]);
}
RSX_F bool any_overflow(const ArenaState& S) {
  uint32_t o = 0;
  for (int i = 0; i < OVF_COUNT; ++i) o |= S.overflow[i];
  return o != 0;
}

// One decision: `n` ticks with `controls` set before each.  Every tick is stepped even after a goal (so that all lanes
// of a warp keep calling the phases together); at the first tick after which the ball is scored, `on_goal(t, S)` gets
// the goal state, which is the decision's result.  Returns the result word without the overflow bit: the scored tick
// (0 none) and kUnimplemented when a tick up to the goal reached a pair the simulator does not implement.
template <class OnGoal, class AfterTick>
RSX_HD inline uint32_t decide(ArenaState& S, const StaticData& D, const Controls* controls, uint32_t n, const OnGoal& on_goal,
                              const AfterTick& after_tick) {
  uint32_t scored = 0, unimpl = 0;
#if defined(__CUDA_ARCH__)
#pragma unroll 1
#endif
  for (uint32_t t = 1; t <= n; ++t) {
    S.cars[0].controls = controls[0];
    S.cars[1].controls = controls[1];
    int st = step_tick(S, D);
    if (scored == 0) {
      if (st != PHASE_OK) unimpl = kUnimplemented;
      after_tick(t, S);
      if (ball_scored(S, D)) {
        scored = t;
        on_goal(t, S);
      }
    }
  }
  return scored | unimpl;
}

struct NoHook {
  RSX_F void operator()(uint32_t, const ArenaState&) const {}
};

// sin(i * 2 pi / 16384), correctly rounded: the auto-flip's 14-bit sine table (StaticData.table_sin)
inline float table_sin_value(int i) {
  int q = i / 4096, k = i % 4096;
  bool swap = k > 2048;
  int kk = swap ? 4096 - k : k;
  crm::U128 r = crm::mulq(crm::small((uint64_t)kk, 124 - 13), crm::kPi[0]);  // kk * pi / 8192
  crm::U128 s, c;
  crm::sincos_fx(r, &s, &c);
  if (swap) {
    crm::U128 t = s;
    s = c;
    c = t;
  }
  crm::U128 v = q == 0 ? s : q == 1 ? c : q == 2 ? crm::neg(s) : crm::neg(c);
  return from_bits(crm::signed_round(v, 0, 0));
}

}  // namespace sim
}  // namespace rsx
