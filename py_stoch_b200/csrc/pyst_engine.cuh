// Per-trajectory simulation engines.
//
// Two mappings of one trajectory onto the GPU:
//   * run_thread<MAXR,...>: one trajectory per thread, for R <= MAXR <= 32.
//     The propensities a[MAXR] live in registers (loops unrolled over the
//     compile-time bound and guarded by j < R); species counts live in a
//     per-thread column of shared memory (element i*bs + lane-of-block).
//   * run_warp<...>: one trajectory per warp, for any R.  Lanes own
//     contiguous reaction slices; the total propensity is a Kogge-Stone
//     prefix sum over the lanes' FP64 partial sums (shuffles) and the firing
//     reaction is found with a ballot over the lane prefixes.
//
// Both restate the reference algorithms:
//   direct method   mod/simulator/cuGillespie/gillespie.py:70-146,
//                   mod/simulator/cuTauLeaping/P3.py:71-151
//   tau-leaping     mod/simulator/cuTauLeaping/P1_P2.py:96-297 with helpers
//                   299-584; the host rounds of cuTauLeaping.py:49-76 become
//                   one loop per trajectory (mode DECIDE = P1_P2, mode SSA =
//                   up to ssa_fallback_steps iterations of P3).
// Precision: propensities FP32; total propensity, clock, cumulative
// selection sums and score integrals FP64; tau selection and leap sampling
// FP32.  Every floating-point operation is explicitly rounded.
#pragma once
#include <stdint.h>

#include "pyst_math.cuh"
#include "pyst_model.cuh"

namespace pyst {

struct RunArgs {
  uint64_t seed;
  int64_t step_budget;
  int32_t ssa_fallback_steps;
  int32_t max_leap_retries;
  int32_t stage_polls;  // bound of the model-staging wait (stage_blob)
};

// Output pointers of one trajectory (already offset to it).
struct TrajOut {
  int32_t* samples;  // element (k*ita + f)*stride
  int64_t stride;
  uint8_t* status;
  int64_t* events;
  uint64_t* seqhash;
  double* t_final;
  double* score;  // [R]
};

#define PYST_I32MAX 2147483647ll
#define PYST_LEAP_TAG 0xFFFFFFFFull

__device__ __forceinline__ float gfun(uint32_t gw, int x) {
  const int H = (int)(gw & 0xFFu);
  const int Ht = (int)((gw >> 8) & 0xFFu);
  const float xf = (float)x;
  if (H == 1) return 1.0f;
  if (H == 2) {
    if (Ht == 2) return __fadd_rn(2.0f, __fdiv_rn(1.0f, __fsub_rn(xf, 1.0f)));
    return 2.0f;
  }
  if (H == 3) {
    if (Ht == 3) {
      const float t1 = __fdiv_rn(1.0f, __fsub_rn(xf, 1.0f));
      const float t2 = __fdiv_rn(2.0f, __fsub_rn(xf, 2.0f));
      return __fadd_rn(__fadd_rn(3.0f, t1), t2);
    }
    if (Ht == 2)
      return __fmul_rn(1.5f,
                       __fadd_rn(2.0f, __fdiv_rn(1.0f, __fsub_rn(xf, 1.0f))));
    return 3.0f;
  }
  if (H >= 4) {
    // Cao-Gillespie-Petzold's g generalised past third order (the
    // reference's CalculateG returns 0 there, P1_P2.py:480-485, which makes
    // tau infinite): g = (H/n) (n + sum_{k=1}^{n-1} k/(x-k)), n = H_type;
    // for H <= 3 this is exactly the table above.
    const int n = Ht < 1 ? 1 : Ht;
    float sm = (float)n;
    for (int k = 1; k < n; ++k)
      sm = __fadd_rn(sm, __fdiv_rn((float)k, __fsub_rn(xf, (float)k)));
    return __fmul_rn(__fdiv_rn((float)H, (float)n), sm);
  }
  return 0.0f;
}

// Candidate tau of one reactant species (P1_P2.py:421-426), FP32.
__device__ __forceinline__ float tau_candidate(float eta, uint32_t gw, int x,
                                               float mu, float s2) {
  const float g = gfun(gw, x);
  const float num = fmaxf(__fdiv_rn(__fmul_rn(eta, (float)x), g), 1.0f);
  const float lhs = __fdiv_rn(num, fabsf(mu));
  const float rhs = __fdiv_rn(__fmul_rn(num, num), s2);
  return fminf(lhs, rhs);
}

__device__ __forceinline__ PoissonKey leap_key(const Stream& s, uint32_t q,
                                               int j, int retry) {
  PoissonKey pk;
  pk.k0 = s.k0;
  pk.k1 = s.k1;
  pk.c0 = q;
  pk.c1 = 0x80000000u | ((uint32_t)j << 12) | ((uint32_t)retry << 6);
  pk.c2 = s.c2;
  pk.c3 = s.c3;
  return pk;
}

// C integer division of two integral FP64 values: the quotient truncated
// toward zero (exact for |a|, |b| < 2^53: a quotient rounded up onto an
// integer is stepped back by the sign of the exact remainder).
__device__ __forceinline__ double law_idiv(double a, double b) {
  if (b == 0.0) return __longlong_as_double(0x7ff8000000000000ll);
  double q = trunc(__ddiv_rn(a, b));
  const double rem = __fma_rn(-q, b, a);
  if (q != 0.0 && rem != 0.0 && ((rem < 0.0) != (a < 0.0)))
    q = __dsub_rn(q, copysign(1.0, q));
  return q;
}

__device__ __forceinline__ double law_exp(double a) {
  if (!(a == a)) return a;
  if (a > 709.0) return __longlong_as_double(0x7ff0000000000000ll);
  if (a < -708.0) return 0.0;
  return pyst_exp(a);
}

__device__ __forceinline__ double law_ln(double a) {
  if (!(a >= 0.0)) return __longlong_as_double(0x7ff8000000000000ll);
  if (a == 0.0) return __longlong_as_double((long long)0xfff0000000000000ull);
  if (a > 1.7976931348623157e308) return a;
  return pyst_log(a);
}

// General kinetic law of reaction j (pyst_model_desc: postfix program over
// the species counts x[i * xs] and FP64 constants), each operation
// explicitly rounded, the result rounded once to the FP32 propensity.  The
// packer checks the programs' stacks; a malformed one gives NaN here (and
// the trajectory the PYST_TRAJ_RATE status).  Out of line: one copy serves
// every call site.
static __device__ __noinline__ float eval_law(const ModelView& m, int j,
                                              const int32_t* x, int xs) {
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  double st[8];
  int sp = 0;
  const int c1 = m.lawptr(j + 1);
  for (int c = m.lawptr(j); c < c1; ++c) {
    const uint32_t wd = m.law(c);
    const int op = (int)(wd >> 24), arg = (int)(wd & 0xFFFFFFu);
    if (op == 1 || op == 2 || op == 16) {
      if (sp >= 8 || (op == 16 && sp < 1)) return (float)nan;
      st[sp] = op == 1 ? (double)x[(int64_t)arg * xs]
                       : (op == 2 ? m.lawc(arg) : st[sp - 1]);
      ++sp;
    } else if (op >= 3 && op <= 7) {
      if (sp < 2) return (float)nan;
      const double b = st[--sp], a = st[sp - 1];
      double r;
      if (op == 3) r = __dadd_rn(a, b);
      else if (op == 4) r = __dsub_rn(a, b);
      else if (op == 5) r = __dmul_rn(a, b);
      else if (op == 6) r = __ddiv_rn(a, b);
      else r = law_idiv(a, b);
      st[sp - 1] = r;
    } else {
      if (sp < 1) return (float)nan;
      const double a = st[sp - 1];
      double r;
      if (op == 8) r = -a;
      else if (op == 10) r = law_exp(a);
      else if (op == 11) r = law_ln(a);
      else if (op == 12) r = __dsqrt_rn(a);
      else if (op == 13) r = fabs(a);
      else if (op == 14) r = floor(a);
      else if (op == 15) r = ceil(a);
      else return (float)nan;
      st[sp - 1] = r;
    }
  }
  return sp == 1 ? __double2float_rn(st[0]) : (float)nan;
}

// A propensity a kinetic law may return: finite and non-negative.
__device__ __forceinline__ bool valid_rate(float a) {
  return a >= 0.0f && a <= 3.4028234663852886e38f;
}

// Propensity of reaction j in FP32: the reaction's kinetic-law program if
// it has one (LAWS: the caller supports them), else the rate, then factors
// in entry order.  Species counts are x[i * xs].
template <bool LAWS = true>
__device__ __forceinline__ float propensity(const ModelView& m, int j,
                                            const int32_t* xc, int xs) {
  if (LAWS && m.nlaw && m.lawptr(j + 1) > m.lawptr(j))
    return eval_law(m, j, xc, xs);
  float a = m.rate(j);
  const int e1 = m.facptr(j + 1);
  for (int e = m.facptr(j); e < e1; ++e) {
    const uint32_t fe = m.fac(e);
    const int x = xc[(int64_t)ent_lo(fe) * xs];
    const int n = fac_order(fe);
    const int fall = fac_falling(fe);
    for (int q = 0; q < n; ++q) a = __fmul_rn(a, (float)(x - q * fall));
  }
  return a;
}

// Packed reaction descriptors for small mass-action reactions, built in
// shared memory by each block after staging the model:
//   factors  pk[j]:     two slots of 13 bits, slot s at bit 13s:
//                       species (10 bits) | order 1..3 (2 bits) | falling
//                       (1 bit); order 0 = empty slot;
//   net      pk[R + j]: two slots of 15 bits, slot s at bit 15s: species
//                       (10 bits) | delta (5-bit two's complement), and the
//                       number of entries in bits 30-31.
// A reaction fits when it has at most two reactant entries of order <= 3
// and at most two net-change entries with |delta| <= 15 over species
// < 1024.  The packed forms take the same operations in the same order as
// the entry lists, so results are identical; they only remove the chains
// of dependent shared-memory loads (entry pointer -> entry -> species).
// Whether reaction j of the blob at `w` fits the packed descriptors: the
// host launchers' form of the conditions pack_reactions checks inline (its
// own form keeps the mode-sorted kernel's register allocation unchanged);
// tests check that both decide alike.
__host__ __device__ inline bool blob_reaction_packable(const uint32_t* w,
                                                       int j) {
  const int ofp = (int)w[PYST_H_OFF_FACPTR], of = (int)w[PYST_H_OFF_FAC];
  const int onp = (int)w[PYST_H_OFF_NETPTR], on = (int)w[PYST_H_OFF_NET];
  const int e0 = (int)w[ofp + j], e1 = (int)w[ofp + j + 1];
  if (e1 - e0 > 2) return false;
  for (int e = e0; e < e1; ++e) {
    const uint32_t fe = w[of + e];
    const int sp = (int)(fe & 0xFFFFu), n = (int)((fe >> 16) & 0xFFu);
    if (sp > 1023 || n < 1 || n > 3) return false;
  }
  const int n0 = (int)w[onp + j], n1 = (int)w[onp + j + 1];
  if (n1 - n0 > 2) return false;
  for (int e = n0; e < n1; ++e) {
    const uint32_t ne = w[on + e];
    const int sp = (int)(ne & 0xFFFFu);
    const int v = (int)(int16_t)(uint16_t)(ne >> 16);
    if (sp > 1023 || v < -16 || v > 15) return false;
  }
  return true;
}

// All threads of the block call this; true when every reaction fits (the
// conditions of blob_reaction_packable, checked inline).
__device__ __forceinline__ bool pack_reactions(const ModelView& m,
                                               uint32_t* pk) {
  bool ok = m.nlaw == 0;  // kinetic-law programs use the general path
  for (int j = threadIdx.x; j < m.R; j += blockDim.x) {
    const int e0 = m.facptr(j), e1 = m.facptr(j + 1);
    uint32_t d = 0;
    if (e1 - e0 > 2) ok = false;
    for (int e = e0; e < e1 && e < e0 + 2; ++e) {
      const uint32_t fe = m.fac(e);
      const int sp = ent_lo(fe), n = fac_order(fe);
      if (sp > 1023 || n < 1 || n > 3) ok = false;
      d |= ((uint32_t)(sp & 1023) | ((uint32_t)(n & 3) << 10) |
            ((uint32_t)fac_falling(fe) << 12))
           << (13 * (e - e0));
    }
    pk[j] = d;
    const int n0 = m.netptr(j), n1 = m.netptr(j + 1);
    uint32_t q = (uint32_t)(n1 - n0) << 30;
    if (n1 - n0 > 2) ok = false;
    for (int e = n0; e < n1 && e < n0 + 2; ++e) {
      const uint32_t ne = m.net(e);
      const int sp = ent_lo(ne), v = ent_hi_s16(ne);
      if (sp > 1023 || v < -16 || v > 15) ok = false;
      q |= ((uint32_t)(sp & 1023) | ((uint32_t)(v & 31) << 10))
           << (15 * (e - n0));
    }
    pk[m.R + j] = q;
  }
  return ok;
}

// propensity() from a packed factor descriptor and the rate.
template <class XGet>
__device__ __forceinline__ float propensity_packed(float rate, uint32_t d,
                                                   XGet xget) {
  float a = rate;
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const uint32_t f = d >> (13 * s);
    const int n = (int)((f >> 10) & 3u);
    if (n) {
      const int x = xget((int)(f & 1023u));
      const int fall = (int)((f >> 12) & 1u);
      a = __fmul_rn(a, (float)x);
      if (n > 1) a = __fmul_rn(a, (float)(x - fall));
      if (n > 2) a = __fmul_rn(a, (float)(x - 2 * fall));
    }
  }
  return a;
}

// Entry q (< 2) of a packed net-change descriptor: species and delta.
__device__ __forceinline__ int pnet_species(uint32_t d, int q) {
  return (int)((d >> (15 * q)) & 1023u);
}
__device__ __forceinline__ int pnet_delta(uint32_t d, int q) {
  return ((int)((d >> (15 * q + 10)) & 31u) ^ 16) - 16;
}
__device__ __forceinline__ int pnet_count(uint32_t d) { return (int)(d >> 30); }

__device__ __forceinline__ void store_sample(const TrajOut& o, int ita, int k,
                                             int f, int32_t v) {
  o.samples[((int64_t)k * ita + f) * o.stride] = v;
}

// ===================================================================
// one trajectory per thread
// ===================================================================
// Everything a thread-mapped trajectory carries between steps, apart from
// its species counts (shared-memory column) and score accumulators.  Split
// out so a block can park a trajectory between scheduling rounds.
struct TState {
  double t;
  uint64_t n;        // Philox block index of the main stream
  int64_t events;
  int64_t steps;
  uint64_t h;        // firing-sequence hash
  int32_t f;         // next sample index
  uint32_t leap_q;   // leaps taken (Poisson stream counter)
  int32_t ssa_left;  // SSA steps left in the current fallback round
  int32_t flags;     // TS_* bits, status in bits 8..15
};

enum {
  TS_SSA = 1,        // in an SSA fallback round (else DECIDE next)
  TS_LEAPGRP = 2,    // last DECIDE chose to leap
  TS_DONE = 4,       // trajectory finished
  TS_FILL = 8        // absorbed: remaining samples take the final state
};

__device__ __forceinline__ int ts_status(const TState& s) {
  return (s.flags >> 8) & 0xFF;
}

template <bool TAU>
__device__ __forceinline__ void thread_init(const ModelView& m, int32_t* xcol,
                                            int bs, TState& s) {
  for (int i = 0; i < m.S; ++i) xcol[(int64_t)i * bs] = m.x0(i);
  s.t = 0.0;
  s.n = 0;
  s.events = 0;
  s.steps = 0;
  s.h = PYST_FNV_OFFSET;
  s.f = 0;
  s.leap_q = 0;
  s.ssa_left = 0;
  s.flags = TAU ? TS_LEAPGRP : TS_SSA;
}

// Advance one trajectory.  Returns when it finishes, or -- for block
// scheduling -- when it has taken cap_ssa SSA steps or cap_leap leaps in
// this call, or when a DECIDE picks the other mode than the one the call
// started in (stop_on_switch).  Species counts are xcol[i*bs], the leap
// scratch of species i is slot[i*ss].  It stops only between steps, so the trajectory resumes
// exactly where it left off.  With unbounded caps this is the whole
// trajectory.
// PK: how reactions are read -- kPkLists (entry lists, general kinetic
// laws included), kPkPacked (packed descriptors, m.fast must hold) or
// kPkRuntime (whichever m.fast says; mass-action models only).
// The fixed forms carry only their own code and live registers (faster for
// the plain kernels); the mode-sorted kernel measured faster with one
// run-time form.
// LG > 1 (direct method only): LG adjacent lanes run the same trajectory
// in lockstep, each on its own species column, and lane g computes the
// Philox block and exponential variate of every LG-th step (g, g + LG, ...);
// a step takes its variates from the owning lane by shuffle.  The random
// numbers, and so the trajectory, are those of LG = 1; only the Philox and
// log work leaves the per-step dependent chain.  The caller lets one lane
// of the group write the outputs.
// GROUP (tau-leaping with stop_on_switch, the mode-sorted scheduler): 0
// any round; kGroupSsa / kGroupLeap when the caller knows the slot's group,
// which lets the compiler drop the code such a round never reaches (an SSA
// round stops when a DECIDE picks a leap, a leap round when it picks SSA
// steps) -- the same arithmetic, a smaller instruction footprint per warp.
enum { kPkLists = 0, kPkPacked = 1, kPkRuntime = 2 };
enum { kGroupAny = 0, kGroupSsa = 1, kGroupLeap = 2 };
// RX: the model's reaction count when the caller fixes it at compile time
// (the per-reaction loops then carry no run-time bound), else 0.
template <int MAXR, bool TAU, bool SCORE, int PK, int LG = 1,
          int GROUP = kGroupAny, int RX = 0>
__device__ void thread_round(const ModelView& m, int32_t* xcol, int64_t* slot,
                             int bs, int ss, const RunArgs& ra,
                             uint64_t traj_id, TState& st, double* integ,
                             int* cnt, const TrajOut& o, int cap_ssa,
                             int cap_leap, bool stop_on_switch) {
  static_assert(RX == 0 || RX == MAXR, "an exact reaction count is MAXR");
  const int S = m.S, R = RX ? RX : m.R, ita = m.ita, kappa = m.kappa;
  const bool pk = PK == kPkPacked || (PK == kPkRuntime && m.fast);
  // general kinetic laws: entry-list form only (a model with laws never
  // packs, and the sorted kernel's run-time form is not given such models)
  constexpr bool kLaws = PK == kPkLists;
#define XV(i) xcol[(int64_t)(i) * bs]
#define SL(i) slot[(int64_t)(i) * ss]
  Stream rs = make_stream(ra.seed, traj_id);
  rs.n = st.n;
  // The main stream is stateless, so its next block (and that block's
  // exponential variate) is computed one step ahead, off the dependent
  // chain of the current step; rs.n runs one block ahead of use.
  static_assert(LG == 1 || (!TAU && LG <= 32 && (LG & (LG - 1)) == 0),
                "lane groups: direct method, power of two up to 32 lanes");
  uint4 w_pf = make_uint4(0u, 0u, 0u, 0u);
  double e_pf = 0.0;
  // lane-group variates: block g_base + g_lane, consumed at step g_i
  const int g_lane = LG > 1 ? (int)(threadIdx.x & (LG - 1)) : 0;
  const unsigned g_mask =
      LG == 32 ? 0xffffffffu
      : LG > 1 ? ((1u << (LG & 31)) - 1u) << (threadIdx.x & 31 & ~(LG - 1))
               : 0u;
  uint64_t g_base = st.n;
  int g_i = 0;
  double g_e = 0.0, g_u = 0.0;
  if constexpr (LG > 1) {
    rs.n = g_base + (uint64_t)g_lane;
    const uint4 wg = next_block(rs);
    g_e = -pyst_log(u53(wg.x, wg.y));
    g_u = u53(wg.z, wg.w);
  } else {
    w_pf = next_block(rs);
    e_pf = -pyst_log(u53(w_pf.x, w_pf.y));
  }
  double t = st.t;
  int f = st.f;
  int64_t events = st.events, steps = st.steps;
  uint64_t h = st.h;
  int status = PYST_TRAJ_DONE;
  bool fill_state = false, done = false;
  const int64_t budget = ra.step_budget;
  const double t_end = m.time(ita - 1);
  double tf = m.time(f);  // next sample time (f < ita while running)
  static_assert(GROUP == kGroupAny || TAU, "groups: tau-leaping only");
  // (a leap-group slot enters in DECIDE mode: the DECIDE that put it there
  // picked a leap)
  bool ssa_mode = GROUP == kGroupLeap ? false : (st.flags & TS_SSA) != 0;
  const bool group_leap = GROUP == kGroupAny ? (st.flags & TS_LEAPGRP) != 0
                                             : GROUP == kGroupLeap;
  bool leap_grp = group_leap;
  int ssa_left = st.ssa_left;
  uint32_t leap_q = st.leap_q;
  int n_ssa = 0, n_leap = 0;
  auto xget = [&](int i) { return XV(i); };

  while (true) {
    // an SSA-group round whose cap falls where a DECIDE is due runs the
    // DECIDE before stopping, so the slot's next round is in the group of
    // its outcome (it would otherwise spend that round only switching).
    // (Leap-group rounds do not: their slots would run every continuing
    // leap's DECIDE twice.)
    const bool capped = n_ssa >= cap_ssa || n_leap >= cap_leap;
    if (capped && !(GROUP == kGroupSsa && !ssa_mode)) break;
    float a[MAXR];
    double a0 = 0.0;
#pragma unroll
    for (int j = 0; j < MAXR; ++j) {
      if (j >= R) break;
      a[j] = pk ? propensity_packed(m.rate(j), m.pk[j], xget)
                    : propensity<kLaws>(m, j, xcol, bs);
      a0 = __dadd_rn(a0, (double)a[j]);
    }
    if (kLaws && m.nlaw) {
      bool bad = false;
#pragma unroll
      for (int j = 0; j < MAXR; ++j) {
        if (j >= R) break;
        bad |= !valid_rate(a[j]);
      }
      if (bad) {
        status = PYST_TRAJ_RATE;
        done = true;
        break;
      }
    }
    if (a0 == 0.0) {
      status = PYST_TRAJ_ABSORBED;
      fill_state = true;
      done = true;
      break;
    }
    if (steps >= budget) {
      status = PYST_TRAJ_STEP_BUDGET;
      done = true;
      break;
    }
    if (TAU && (GROUP == kGroupLeap || !ssa_mode)) {
      // ---------------- DECIDE: critical set, tau_1, SSA switch -------
      uint32_t crit = 0u;
#pragma unroll
      for (int j = 0; j < MAXR; ++j) {
        if (j >= R) break;
        if (pk) {
          // the negative entries of the net change (same test, any order)
          const uint32_t d = m.pk[R + j];
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int v = pnet_delta(d, q);
            if (q < pnet_count(d) && v < 0 &&
                (int64_t)(-v) * m.n_c > (int64_t)XV(pnet_species(d, q)))
              crit |= 1u << j;
          }
        } else {
          const int e1 = m.critptr(j + 1);
          for (int e = m.critptr(j); e < e1; ++e) {
            const uint32_t ce = m.crit(e);
            if ((int64_t)(ce >> 16) * m.n_c > (int64_t)XV(ent_lo(ce)))
              crit |= 1u << j;
          }
        }
      }
      for (int i = 0; i < S; ++i) SL(i) = 0;
#pragma unroll
      for (int j = 0; j < MAXR; ++j) {
        if (j >= R) break;
        if (!((crit >> j) & 1u)) {
          auto acc = [&](int sp, int v) {
            float2 ms = *reinterpret_cast<float2*>(&SL(sp));
            ms.x = __fadd_rn(ms.x, __fmul_rn((float)v, a[j]));
            ms.y = __fadd_rn(ms.y, __fmul_rn((float)(v * v), a[j]));
            *reinterpret_cast<float2*>(&SL(sp)) = ms;
          };
          if (pk) {
            const uint32_t d = m.pk[R + j];
#pragma unroll
            for (int q = 0; q < 2; ++q)
              if (q < pnet_count(d)) acc(pnet_species(d, q), pnet_delta(d, q));
          } else {
            const int e1 = m.netptr(j + 1);
            for (int e = m.netptr(j); e < e1; ++e) {
              const uint32_t ne = m.net(e);
              acc(ent_lo(ne), ent_hi_s16(ne));
            }
          }
        }
      }
      float tau1 = __int_as_float(0x7f800000);
      for (int i = 0; i < S; ++i) {
        const uint32_t gw = m.g(i);
        if (!((gw >> 16) & 1u)) continue;
        const float2 ms = *reinterpret_cast<float2*>(&SL(i));
        const float c = tau_candidate(m.eta, gw, XV(i), ms.x, ms.y);
        if (c < tau1) tau1 = c;
      }
      if ((double)tau1 < __ddiv_rn(10.0, a0)) {
        ssa_mode = true;
        ssa_left = ra.ssa_fallback_steps;
        leap_grp = false;
        // regroup before stepping
        if (capped || GROUP == kGroupLeap || (stop_on_switch && group_leap))
          break;
        // fall through to the SSA step below with the same propensities
      } else {
        leap_grp = true;
        if (capped || GROUP == kGroupSsa || (stop_on_switch && !group_leap))
          break;
        // ---------------- leap ---------------------------------------
        steps++;
        n_leap++;
        double a0c = 0.0;
#pragma unroll
        for (int j = 0; j < MAXR; ++j) {
          if (j >= R) break;
          if ((crit >> j) & 1u) a0c = __dadd_rn(a0c, (double)a[j]);
        }
        double tau2 = __longlong_as_double(0x7ff0000000000000ll);
        uint4 wc = make_uint4(0, 0, 0, 0);
        if (a0c > 0.0) {
          wc = w_pf;
          tau2 = __ddiv_rn(e_pf, a0c);
          w_pf = next_block(rs);
          e_pf = -pyst_log(u53(w_pf.x, w_pf.y));
        }
        const double tau1d = (double)tau1;
        double tau = (tau2 < tau1d) ? tau2 : tau1d;
        int kcrit = -1;
        if (tau1d > tau2) {
          const double r = __dmul_rn(u53(wc.z, wc.w), a0c);
          double cum = 0.0;
          int lastnz = -1;
#pragma unroll
          for (int j = 0; j < MAXR; ++j) {
            if (j >= R) break;
            if ((crit >> j) & 1u) {
              cum = __dadd_rn(cum, (double)a[j]);
              if (a[j] > 0.0f) lastnz = j;
              if (cum >= r) {
                kcrit = j;
                break;
              }
            }
          }
          if (kcrit < 0) kcrit = lastnz;
        }
        int K[MAXR];
        int retry = 0;
        bool ok = false;
        while (true) {
          bool bad = false;
          auto draw = [&](int j, float aj) {
            if ((crit >> j) & 1u) return (j == kcrit) ? 1 : 0;
            const float lam = __fmul_rn(aj, (float)tau);
            const int k = poisson(lam, leap_key(rs, leap_q, j, retry));
            if (k < 0) bad = true;
            return k < 0 ? 0 : k;
          };
          if constexpr (GROUP != kGroupAny && RX == 0) {
            // (the mode-sorted scheduler's leap rounds with a run-time
            // reaction count) one reaction per iteration, not unrolled: a
            // single inlined copy of the sampler's call sequence, a[j] and
            // K[j] by unrolled selects.  With the count fixed at compile
            // time the unrolled loop below measured as fast or faster
            // (6-reaction network 11.6 vs 12.0 ms).
#pragma unroll 1
            for (int j = 0; j < R; ++j) {
              float aj = a[0];
#pragma unroll
              for (int q = 1; q < MAXR; ++q) aj = (j == q) ? a[q] : aj;
              const int kj = draw(j, aj);
#pragma unroll
              for (int q = 0; q < MAXR; ++q)
                if (q == j) K[q] = kj;
            }
          } else {
#pragma unroll
            for (int j = 0; j < MAXR; ++j) {
              if (j >= R) break;
              K[j] = draw(j, a[j]);
            }
          }
          if (bad) {
            status = PYST_TRAJ_SAMPLER;
            break;
          }
          for (int i = 0; i < S; ++i) SL(i) = 0;
#pragma unroll
          for (int j = 0; j < MAXR; ++j) {
            if (j >= R) break;
            if (K[j] != 0) {
              if (pk) {
                const uint32_t d = m.pk[R + j];
#pragma unroll
                for (int q = 0; q < 2; ++q)
                  if (q < pnet_count(d))
                    SL(pnet_species(d, q)) += (int64_t)K[j] * pnet_delta(d, q);
              } else {
                const int e1 = m.netptr(j + 1);
                for (int e = m.netptr(j); e < e1; ++e) {
                  const uint32_t ne = m.net(e);
                  SL(ent_lo(ne)) += (int64_t)K[j] * ent_hi_s16(ne);
                }
              }
            }
          }
          bool neg = false, over = false;
          for (int i = 0; i < S; ++i) {
            const int64_t nx = (int64_t)XV(i) + SL(i);
            neg |= nx < 0;
            over |= nx > PYST_I32MAX;
          }
          if (over) {
            status = PYST_TRAJ_OVERFLOW;
            break;
          }
          if (!neg) {
            ok = true;
            break;
          }
          tau = __dmul_rn(tau, 0.5);
          retry++;
          if (retry > ra.max_leap_retries) {
            status = PYST_TRAJ_LEAP_RETRY;
            break;
          }
        }
        if (!ok) {
          done = true;
          break;
        }
        leap_q++;
        const double tn = __dadd_rn(t, tau);
        int64_t fired = 0;
        h = seq_mix(h, PYST_LEAP_TAG);
#pragma unroll
        for (int j = 0; j < MAXR; ++j) {
          if (j >= R) break;
          fired += K[j];
          if (K[j] != 0) h = seq_mix(h, ((uint64_t)j << 32) | (uint32_t)K[j]);
          if (SCORE) {
            cnt[j] += K[j];
            integ[j] = __dadd_rn(integ[j], __dmul_rn((double)a[j], tau));
          }
        }
        while (tn >= tf) {
          const double frac = __ddiv_rn(__dsub_rn(tf, t), tau);
          for (int k = 0; k < kappa; ++k) {
            const int i = m.out(k);
            const double inc = rint(__dmul_rn((double)SL(i), frac));
            store_sample(o, ita, k, f, XV(i) + (int)inc);
          }
          f++;
          if (f == ita) {
            done = true;
            break;
          }
          tf = m.time(f);
        }
        for (int i = 0; i < S; ++i) XV(i) = (int)((int64_t)XV(i) + SL(i));
        events += fired;
        t = tn;
        if (done) break;
        continue;
      }
    }
    // ------------------------ one direct-method step -------------------
    steps++;
    n_ssa++;
    double tau, r;
    if constexpr (LG > 1) {
      const double e = __shfl_sync(g_mask, g_e, g_i, LG);
      const double uu = __shfl_sync(g_mask, g_u, g_i, LG);
      tau = __ddiv_rn(e, a0);
      r = __dmul_rn(uu, a0);
      if (++g_i == LG) {
        g_i = 0;
        g_base += LG;
        rs.n = g_base + (uint64_t)g_lane;
        const uint4 wg = next_block(rs);
        g_e = -pyst_log(u53(wg.x, wg.y));
        g_u = u53(wg.z, wg.w);
      }
    } else {
      const uint4 w = w_pf;
      tau = __ddiv_rn(e_pf, a0);
      w_pf = next_block(rs);
      e_pf = -pyst_log(u53(w_pf.x, w_pf.y));
      r = __dmul_rn(u53(w.z, w.w), a0);
    }
    int sel = -1;
    {
      double cum = 0.0;
      int lastnz = -1;
#pragma unroll
      for (int j = 0; j < MAXR; ++j) {
        if (j >= R) break;
        cum = __dadd_rn(cum, (double)a[j]);
        if (a[j] > 0.0f) lastnz = j;
        if (cum >= r) {
          sel = j;
          break;
        }
      }
      // unreachable in exact arithmetic (the last sum equals a0 >= r);
      // kept so a selection always names a reaction with a_j > 0
      if (sel < 0) sel = lastnz;
    }
    const double tn = __dadd_rn(t, tau);
    if (SCORE) {
      const double dt = (tn >= t_end) ? __dsub_rn(t_end, t) : tau;
#pragma unroll
      for (int j = 0; j < MAXR; ++j) {
        if (j >= R) break;
        integ[j] = __dadd_rn(integ[j], __dmul_rn((double)a[j], dt));
      }
    }
    while (tn >= tf) {
      if (LG == 1 || g_lane == 0)
        for (int k = 0; k < kappa; ++k)
          store_sample(o, ita, k, f, XV(m.out(k)));
      f++;
      if (f == ita) {
        done = true;
        break;
      }
      tf = m.time(f);
    }
    t = tn;
    if (done) break;
    {
      bool over = false;
      if (pk) {
        const uint32_t d = m.pk[R + sel];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          if (q < pnet_count(d)) {
            const int sp = pnet_species(d, q);
            const int64_t nx = (int64_t)XV(sp) + pnet_delta(d, q);
            if (nx < 0 || nx > PYST_I32MAX) over = true;
            else XV(sp) = (int)nx;
          }
        }
      } else {
        const int e1 = m.netptr(sel + 1);
        for (int e = m.netptr(sel); e < e1; ++e) {
          const uint32_t ne = m.net(e);
          const int sp = ent_lo(ne);
          const int64_t nx = (int64_t)XV(sp) + ent_hi_s16(ne);
          if (nx < 0 || nx > PYST_I32MAX) over = true;
          else XV(sp) = (int)nx;
        }
      }
      if (over) {
        status = PYST_TRAJ_OVERFLOW;
        done = true;
        break;
      }
    }
    events++;
    h = seq_mix(h, (uint64_t)sel);
    if (SCORE) {
#pragma unroll
      for (int j = 0; j < MAXR; ++j) cnt[j] += (j == sel) ? 1 : 0;
    }
    if (TAU) {
      if (--ssa_left <= 0) ssa_mode = false;
    }
  }
  st.t = t;
  // the prefetched block (LG = 1) was not used
  st.n = LG > 1 ? g_base + (uint64_t)g_i : rs.n - 1;
  st.events = events;
  st.steps = steps;
  st.h = h;
  st.f = f;
  st.leap_q = leap_q;
  st.ssa_left = ssa_left;
  st.flags = (ssa_mode ? TS_SSA : 0) | (leap_grp ? TS_LEAPGRP : 0) |
             (done ? TS_DONE : 0) | (fill_state ? TS_FILL : 0) |
             (status << 8);
#undef XV
#undef SL
}

// Write the remaining samples (state after absorption, -1 after an error)
// and the per-trajectory outputs of a finished trajectory.
template <int MAXR, bool SCORE>
__device__ void thread_finish(const ModelView& m, const int32_t* xcol, int bs,
                              const TState& st, const double* integ,
                              const int* cnt, const TrajOut& o) {
  const int ita = m.ita, kappa = m.kappa, R = m.R;
  const bool fill_state = (st.flags & TS_FILL) != 0;
  for (int f = st.f; f < ita; ++f)
    for (int k = 0; k < kappa; ++k)
      store_sample(o, ita, k, f,
                   fill_state ? xcol[(int64_t)m.out(k) * bs] : -1);
  if (o.status) *o.status = (uint8_t)ts_status(st);
  if (o.events) *o.events = st.events;
  if (o.seqhash) *o.seqhash = st.h;
  if (o.t_final) *o.t_final = st.t;
  if (SCORE && o.score) {
#pragma unroll
    for (int j = 0; j < MAXR; ++j) {
      if (j >= R) break;
      o.score[j] = __dsub_rn((double)cnt[j], integ[j]);
    }
  }
}

// One whole trajectory by the calling thread.  PK: kPkPacked or kPkLists
// when the caller knows the form (the host checks packability), -1 to
// choose by m.fast at run time (batched launches mix models).
// RX as thread_round's.
template <int MAXR, bool TAU, bool SCORE, int PK = -1, int RX = 0>
__device__ void run_thread(const ModelView& m, int32_t* xcol, int64_t* slot,
                           int bs, const RunArgs& ra, uint64_t traj_id,
                           const TrajOut& o) {
  TState st;
  thread_init<TAU>(m, xcol, bs, st);
  double integ[SCORE ? MAXR : 1];
  int cnt[SCORE ? MAXR : 1];
#pragma unroll
  for (int j = 0; j < (SCORE ? MAXR : 1); ++j) {
    integ[j] = 0.0;
    cnt[j] = 0;
  }
  if (PK == kPkPacked || (PK < 0 && m.fast))
    thread_round<MAXR, TAU, SCORE, kPkPacked, 1, kGroupAny, RX>(
        m, xcol, slot, bs, bs, ra, traj_id, st, integ, cnt, o, 0x7fffffff,
        0x7fffffff, false);
  else if (PK == kPkLists || PK < 0)
    thread_round<MAXR, TAU, SCORE, kPkLists, 1, kGroupAny, RX>(
        m, xcol, slot, bs, bs, ra, traj_id, st, integ, cnt, o, 0x7fffffff,
        0x7fffffff, false);
  thread_finish<MAXR, SCORE>(m, xcol, bs, st, integ, cnt, o);
}

// ===================================================================
// one trajectory per thread, any number of reactions
// ===================================================================
// Same steps and arithmetic as thread_round, for R beyond the register
// arrays: loops over reactions are not unrolled and propensities are
// recomputed where thread_round reads a[j] again (selection pass, critical
// sums, leap means), so nothing per reaction is stored.  The critical flag
// of a reaction is re-derived from the species counts when needed.
__device__ __forceinline__ bool is_critical(const ModelView& m, int j,
                                            const int32_t* xcol, int bs) {
  const int e1 = m.critptr(j + 1);
  for (int e = m.critptr(j); e < e1; ++e) {
    const uint32_t ce = m.crit(e);
    if ((int64_t)(ce >> 16) * m.n_c >
        (int64_t)xcol[(int64_t)ent_lo(ce) * bs])
      return true;
  }
  return false;
}

template <bool TAU>
__device__ void thread_round_big(const ModelView& m, int32_t* xcol,
                                 int64_t* slot, int bs, int ss,
                                 const RunArgs& ra, uint64_t traj_id,
                                 TState& st, const TrajOut& o, int cap_ssa,
                                 int cap_leap, bool stop_on_switch) {
  const int S = m.S, R = m.R, ita = m.ita, kappa = m.kappa;
#define XV(i) xcol[(int64_t)(i) * bs]
#define SL(i) slot[(int64_t)(i) * ss]
  Stream rs = make_stream(ra.seed, traj_id);
  rs.n = st.n;
  double t = st.t;
  int f = st.f;
  int64_t events = st.events, steps = st.steps;
  uint64_t h = st.h;
  int status = PYST_TRAJ_DONE;
  bool fill_state = false, done = false;
  const int64_t budget = ra.step_budget;
  bool ssa_mode = (st.flags & TS_SSA) != 0;
  const bool group_leap = (st.flags & TS_LEAPGRP) != 0;
  bool leap_grp = group_leap;
  int ssa_left = st.ssa_left;
  uint32_t leap_q = st.leap_q;
  int n_ssa = 0, n_leap = 0;
  auto xget = [&](int i) { return XV(i); };

  while (true) {
    if (n_ssa >= cap_ssa || n_leap >= cap_leap) break;
    double a0 = 0.0;
    bool bad_rate = false;
    for (int j = 0; j < R; ++j) {
      const float aj = propensity(m, j, xcol, bs);
      bad_rate |= !valid_rate(aj);
      a0 = __dadd_rn(a0, (double)aj);
    }
    if (m.nlaw && bad_rate) {
      status = PYST_TRAJ_RATE;
      done = true;
      break;
    }
    if (a0 == 0.0) {
      status = PYST_TRAJ_ABSORBED;
      fill_state = true;
      done = true;
      break;
    }
    if (steps >= budget) {
      status = PYST_TRAJ_STEP_BUDGET;
      done = true;
      break;
    }
    if (TAU && !ssa_mode) {
      for (int i = 0; i < S; ++i) SL(i) = 0;
      for (int j = 0; j < R; ++j) {
        if (is_critical(m, j, xcol, bs)) continue;
        const float aj = propensity(m, j, xcol, bs);
        const int e1 = m.netptr(j + 1);
        for (int e = m.netptr(j); e < e1; ++e) {
          const uint32_t ne = m.net(e);
          const int sp = ent_lo(ne);
          const int v = ent_hi_s16(ne);
          float2 ms = *reinterpret_cast<float2*>(&SL(sp));
          ms.x = __fadd_rn(ms.x, __fmul_rn((float)v, aj));
          ms.y = __fadd_rn(ms.y, __fmul_rn((float)(v * v), aj));
          *reinterpret_cast<float2*>(&SL(sp)) = ms;
        }
      }
      float tau1 = __int_as_float(0x7f800000);
      for (int i = 0; i < S; ++i) {
        const uint32_t gw = m.g(i);
        if (!((gw >> 16) & 1u)) continue;
        const float2 ms = *reinterpret_cast<float2*>(&SL(i));
        const float c = tau_candidate(m.eta, gw, XV(i), ms.x, ms.y);
        if (c < tau1) tau1 = c;
      }
      if ((double)tau1 < __ddiv_rn(10.0, a0)) {
        ssa_mode = true;
        ssa_left = ra.ssa_fallback_steps;
        leap_grp = false;
        if (stop_on_switch && group_leap) break;
      } else {
        leap_grp = true;
        if (stop_on_switch && !group_leap) break;
        steps++;
        n_leap++;
        double a0c = 0.0;
        for (int j = 0; j < R; ++j)
          if (is_critical(m, j, xcol, bs))
            a0c = __dadd_rn(a0c, (double)propensity(m, j, xcol, bs));
        double tau2 = __longlong_as_double(0x7ff0000000000000ll);
        uint4 wc = make_uint4(0, 0, 0, 0);
        if (a0c > 0.0) {
          wc = next_block(rs);
          tau2 = __ddiv_rn(-pyst_log(u53(wc.x, wc.y)), a0c);
        }
        const double tau1d = (double)tau1;
        double tau = (tau2 < tau1d) ? tau2 : tau1d;
        int kcrit = -1;
        if (tau1d > tau2) {
          const double r = __dmul_rn(u53(wc.z, wc.w), a0c);
          double cum = 0.0;
          int lastnz = -1;
          for (int j = 0; j < R; ++j) {
            if (!is_critical(m, j, xcol, bs)) continue;
            const float aj = propensity(m, j, xcol, bs);
            cum = __dadd_rn(cum, (double)aj);
            if (aj > 0.0f) lastnz = j;
            if (cum >= r) {
              kcrit = j;
              break;
            }
          }
          if (kcrit < 0) kcrit = lastnz;
        }
        int retry = 0;
        bool ok = false;
        int64_t fired = 0;
        uint64_t hl = 0;
        while (true) {
          // Poisson firings, accumulated straight into the state change
          for (int i = 0; i < S; ++i) SL(i) = 0;
          bool bad = false;
          fired = 0;
          hl = seq_mix(h, PYST_LEAP_TAG);
          for (int j = 0; j < R; ++j) {
            int kj;
            if (is_critical(m, j, xcol, bs)) {
              kj = (j == kcrit) ? 1 : 0;
            } else {
              const float lam =
                  __fmul_rn(propensity(m, j, xcol, bs), (float)tau);
              const int k = poisson(lam, leap_key(rs, leap_q, j, retry));
              if (k < 0) bad = true;
              kj = k < 0 ? 0 : k;
            }
            if (kj != 0) {
              fired += kj;
              hl = seq_mix(hl, ((uint64_t)j << 32) | (uint32_t)kj);
              const int e1 = m.netptr(j + 1);
              for (int e = m.netptr(j); e < e1; ++e) {
                const uint32_t ne = m.net(e);
                SL(ent_lo(ne)) += (int64_t)kj * ent_hi_s16(ne);
              }
            }
          }
          if (bad) {
            status = PYST_TRAJ_SAMPLER;
            break;
          }
          bool neg = false, over = false;
          for (int i = 0; i < S; ++i) {
            const int64_t nx = (int64_t)XV(i) + SL(i);
            neg |= nx < 0;
            over |= nx > PYST_I32MAX;
          }
          if (over) {
            status = PYST_TRAJ_OVERFLOW;
            break;
          }
          if (!neg) {
            ok = true;
            break;
          }
          tau = __dmul_rn(tau, 0.5);
          retry++;
          if (retry > ra.max_leap_retries) {
            status = PYST_TRAJ_LEAP_RETRY;
            break;
          }
        }
        if (!ok) {
          done = true;
          break;
        }
        leap_q++;
        h = hl;
        const double tn = __dadd_rn(t, tau);
        while (tn >= m.time(f)) {
          const double frac = __ddiv_rn(__dsub_rn(m.time(f), t), tau);
          for (int k = 0; k < kappa; ++k) {
            const int i = m.out(k);
            const double inc = rint(__dmul_rn((double)SL(i), frac));
            store_sample(o, ita, k, f, XV(i) + (int)inc);
          }
          f++;
          if (f == ita) {
            done = true;
            break;
          }
        }
        for (int i = 0; i < S; ++i) XV(i) = (int)((int64_t)XV(i) + SL(i));
        events += fired;
        t = tn;
        if (done) break;
        continue;
      }
    }
    // ------------------------ one direct-method step -------------------
    steps++;
    n_ssa++;
    const uint4 w = next_block(rs);
    const double tau = __ddiv_rn(-pyst_log(u53(w.x, w.y)), a0);
    const double r = __dmul_rn(u53(w.z, w.w), a0);
    int sel = -1;
    {
      double cum = 0.0;
      int lastnz = -1;
      for (int j = 0; j < R; ++j) {
        const float aj = propensity(m, j, xcol, bs);
        cum = __dadd_rn(cum, (double)aj);
        if (aj > 0.0f) lastnz = j;
        if (cum >= r) {
          sel = j;
          break;
        }
      }
      if (sel < 0) sel = lastnz;
    }
    const double tn = __dadd_rn(t, tau);
    while (tn >= m.time(f)) {
      for (int k = 0; k < kappa; ++k) store_sample(o, ita, k, f, XV(m.out(k)));
      f++;
      if (f == ita) {
        done = true;
        break;
      }
    }
    t = tn;
    if (done) break;
    {
      const int e1 = m.netptr(sel + 1);
      bool over = false;
      for (int e = m.netptr(sel); e < e1; ++e) {
        const uint32_t ne = m.net(e);
        const int sp = ent_lo(ne);
        const int64_t nx = (int64_t)XV(sp) + ent_hi_s16(ne);
        if (nx < 0 || nx > PYST_I32MAX) over = true;
        else XV(sp) = (int)nx;
      }
      if (over) {
        status = PYST_TRAJ_OVERFLOW;
        done = true;
        break;
      }
    }
    events++;
    h = seq_mix(h, (uint64_t)sel);
    if (TAU) {
      if (--ssa_left <= 0) ssa_mode = false;
    }
  }
  st.t = t;
  st.n = rs.n;
  st.events = events;
  st.steps = steps;
  st.h = h;
  st.f = f;
  st.leap_q = leap_q;
  st.ssa_left = ssa_left;
  st.flags = (ssa_mode ? TS_SSA : 0) | (leap_grp ? TS_LEAPGRP : 0) |
             (done ? TS_DONE : 0) | (fill_state ? TS_FILL : 0) |
             (status << 8);
#undef XV
#undef SL
}

// thread_round for MAXR > 0 (register arrays), thread_round_big for 0; PK,
// GROUP and RX as thread_round's
template <int MAXR, bool TAU, bool SCORE, int PK = kPkRuntime,
          int GROUP = kGroupAny, int RX = 0>
__device__ __forceinline__ void any_round(
    const ModelView& m, int32_t* xcol, int64_t* slot, int bs, int ss,
    const RunArgs& ra, uint64_t traj_id, TState& st, double* integ, int* cnt,
    const TrajOut& o, int cap_ssa, int cap_leap, bool stop_on_switch) {
  if constexpr (MAXR == 0) {
    static_assert(!SCORE, "the large-R thread engine keeps no scores");
    thread_round_big<TAU>(m, xcol, slot, bs, ss, ra, traj_id, st, o, cap_ssa,
                          cap_leap, stop_on_switch);
  } else {
    thread_round<MAXR, TAU, SCORE, PK, 1, GROUP, RX>(
        m, xcol, slot, bs, ss, ra, traj_id, st, integ, cnt, o, cap_ssa,
        cap_leap, stop_on_switch);
  }
}

template <bool TAU>
__device__ void run_thread_big(const ModelView& m, int32_t* xcol,
                               int64_t* slot, int bs, const RunArgs& ra,
                               uint64_t traj_id, const TrajOut& o) {
  TState st;
  thread_init<TAU>(m, xcol, bs, st);
  thread_round_big<TAU>(m, xcol, slot, bs, bs, ra, traj_id, st, o,
                        0x7fffffff, 0x7fffffff, false);
  thread_finish<1, false>(m, xcol, bs, st, nullptr, nullptr, o);
}

// ===================================================================
// one trajectory per warp
// ===================================================================
// Per-warp shared memory: x[S] int32, a[R] float, slot[S] 8 bytes,
// K[R] int32, crit[R] uint8 (rounded up to 4).  Lane l owns reactions
// [l*c, min(R,(l+1)*c)) with c = ceil(R/32); it owns species l, l+32, ...
struct WarpSmem {
  int32_t* x;
  float* a;
  int64_t* slot;
  int32_t* K;
  uint8_t* crit;
};

__device__ __forceinline__ size_t warp_smem_bytes(int S, int R) {
  size_t b = (size_t)S * 8 + (size_t)S * 4 + (size_t)R * 4 + (size_t)R * 4 +
             (((size_t)R + 3) & ~(size_t)3);
  return (b + 15) & ~(size_t)15;
}

__device__ __forceinline__ WarpSmem warp_smem(void* base, int S, int R) {
  WarpSmem w;
  char* p = (char*)base;
  w.slot = (int64_t*)p;
  p += (size_t)S * 8;
  w.x = (int32_t*)p;
  p += (size_t)S * 4;
  w.a = (float*)p;
  p += (size_t)R * 4;
  w.K = (int32_t*)p;
  p += (size_t)R * 4;
  w.crit = (uint8_t*)p;
  return w;
}

// Kogge-Stone inclusive scan of lane partial sums (FP64).  The oracle's
// warp mode repeats exactly these additions.
__device__ __forceinline__ double warp_incl_scan(double v, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double n = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v = __dadd_rn(n, v);
  }
  return v;
}

// Select within lane prefixes: first lane L with p_L > 0 and incl_L >= r
// (fallback: last lane with p > 0); inside L, with r' = r - (incl_L - p_L),
// the first owned j whose running sum reaches r' (fallback: last owned j
// with a_j > 0).  Returns j on every lane.
__device__ __forceinline__ int warp_select(const float* a, double part,
                                          double incl, double r, int j0,
                                          int j1, int lane,
                                          const uint8_t* mask) {
  const unsigned hit = __ballot_sync(0xffffffffu, part > 0.0 && incl >= r);
  const unsigned nz = __ballot_sync(0xffffffffu, part > 0.0);
  const int L = hit ? (__ffs(hit) - 1) : (31 - __clz(nz));
  int sel = -1;
  if (lane == L) {
    const double rr = __dsub_rn(r, __dsub_rn(incl, part));
    double cum = 0.0;
    int lastnz = -1;
    for (int j = j0; j < j1; ++j) {
      if (mask && !mask[j]) continue;
      const float aj = a[j];
      cum = __dadd_rn(cum, (double)aj);
      if (aj > 0.0f) lastnz = j;
      if (cum >= rr) {
        sel = j;
        break;
      }
    }
    if (sel < 0) sel = lastnz;
  }
  return __shfl_sync(0xffffffffu, sel, L);
}

template <bool TAU, bool SCORE>
__device__ void run_warp(const ModelView& m, const WarpSmem& ws,
                         const RunArgs& ra, uint64_t traj_id, const TrajOut& o,
                         double* score_acc /* per-warp [R] or null */) {
  const int S = m.S, R = m.R, ita = m.ita, kappa = m.kappa;
  const int lane = threadIdx.x & 31;
  const int c = (R + 31) >> 5;
  const int j0 = min(R, lane * c), j1 = min(R, j0 + c);
  for (int i = lane; i < S; i += 32) ws.x[i] = m.x0(i);
  if (SCORE)
    for (int j = lane; j < 2 * R; j += 32) score_acc[j] = 0.0;
  __syncwarp();
  Stream rs = make_stream(ra.seed, traj_id);
  double t = 0.0;
  int f = 0;
  int64_t events = 0, steps = 0;
  uint64_t h = PYST_FNV_OFFSET;
  int status = PYST_TRAJ_DONE;
  bool fill_state = false;
  const double t_end = m.time(ita - 1);
  bool ssa_mode = !TAU;
  int ssa_left = 0;
  uint32_t leap_q = 0;
  auto xget = [&](int i) { return ws.x[i]; };

  while (true) {
    double part = 0.0;
    bool bad_rate = false;
    for (int j = j0; j < j1; ++j) {
      const float aj = propensity(m, j, ws.x, 1);
      bad_rate |= !valid_rate(aj);
      ws.a[j] = aj;
      part = __dadd_rn(part, (double)aj);
    }
    const double incl = warp_incl_scan(part, lane);
    const double a0 = __shfl_sync(0xffffffffu, incl, 31);
    __syncwarp();
    if (__any_sync(0xffffffffu, m.nlaw && bad_rate)) {
      status = PYST_TRAJ_RATE;
      break;
    }
    if (a0 == 0.0) {
      status = PYST_TRAJ_ABSORBED;
      fill_state = true;
      break;
    }
    if (steps >= ra.step_budget) {
      status = PYST_TRAJ_STEP_BUDGET;
      break;
    }
    if (TAU && !ssa_mode) {
      // critical flags for owned reactions
      for (int j = j0; j < j1; ++j) {
        uint8_t cf = 0;
        const int e1 = m.critptr(j + 1);
        for (int e = m.critptr(j); e < e1; ++e) {
          const uint32_t ce = m.crit(e);
          if ((int64_t)(ce >> 16) * m.n_c > (int64_t)ws.x[ent_lo(ce)]) cf = 1;
        }
        ws.crit[j] = cf;
      }
      __syncwarp();
      // mu, sigma^2 and the tau candidate per owned species
      float tmin = __int_as_float(0x7f800000);
      for (int i = lane; i < S; i += 32) {
        const uint32_t gw = m.g(i);
        if (!((gw >> 16) & 1u)) continue;
        float mu = 0.0f, s2 = 0.0f;
        const int e1 = m.spvptr(i + 1);
        for (int e = m.spvptr(i); e < e1; ++e) {
          const uint32_t se = m.spv(e);
          const int j = ent_lo(se);
          if (ws.crit[j]) continue;
          const int v = ent_hi_s16(se);
          mu = __fadd_rn(mu, __fmul_rn((float)v, ws.a[j]));
          s2 = __fadd_rn(s2, __fmul_rn((float)(v * v), ws.a[j]));
        }
        const float cnd = tau_candidate(m.eta, gw, ws.x[i], mu, s2);
        if (cnd < tmin) tmin = cnd;
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1)
        tmin = fminf(tmin, __shfl_xor_sync(0xffffffffu, tmin, d));
      const float tau1 = tmin;
      if ((double)tau1 < __ddiv_rn(10.0, a0)) {
        ssa_mode = true;
        ssa_left = ra.ssa_fallback_steps;
      } else {
        steps++;
        double pc = 0.0;
        for (int j = j0; j < j1; ++j)
          if (ws.crit[j]) pc = __dadd_rn(pc, (double)ws.a[j]);
        const double inc_c = warp_incl_scan(pc, lane);
        const double a0c = __shfl_sync(0xffffffffu, inc_c, 31);
        double tau2 = __longlong_as_double(0x7ff0000000000000ll);
        uint4 wc = make_uint4(0, 0, 0, 0);
        if (a0c > 0.0) {
          wc = next_block(rs);
          tau2 = __ddiv_rn(-pyst_log(u53(wc.x, wc.y)), a0c);
        }
        const double tau1d = (double)tau1;
        double tau = (tau2 < tau1d) ? tau2 : tau1d;
        int kcrit = -1;
        if (tau1d > tau2) {
          const double r = __dmul_rn(u53(wc.z, wc.w), a0c);
          kcrit = warp_select(ws.a, pc, inc_c, r, j0, j1, lane, ws.crit);
        }
        int retry = 0;
        bool ok = false;
        while (true) {
          bool bad = false;
          for (int j = j0; j < j1; ++j) {
            int kj = 0;
            if (ws.crit[j]) {
              kj = (j == kcrit) ? 1 : 0;
            } else {
              const float lam = __fmul_rn(ws.a[j], (float)tau);
              const int k = poisson(lam, leap_key(rs, leap_q, j, retry));
              if (k < 0) bad = true;
              kj = k < 0 ? 0 : k;
            }
            ws.K[j] = kj;
          }
          for (int i = lane; i < S; i += 32) ws.slot[i] = 0;
          __syncwarp();
          if (__any_sync(0xffffffffu, bad)) {
            status = PYST_TRAJ_SAMPLER;
            break;
          }
          // species-major accumulation of V K (lane owns species)
          bool neg = false, over = false;
          for (int i = lane; i < S; i += 32) {
            int64_t d = 0;
            const int e1 = m.spvptr(i + 1);
            const uint32_t gw = m.g(i);
            (void)gw;
            for (int e = m.spvptr(i); e < e1; ++e) {
              const uint32_t se = m.spv(e);
              d += (int64_t)ws.K[ent_lo(se)] * ent_hi_s16(se);
            }
            ws.slot[i] = d;
            const int64_t nx = (int64_t)ws.x[i] + d;
            neg |= nx < 0;
            over |= nx > PYST_I32MAX;
          }
          __syncwarp();
          if (__any_sync(0xffffffffu, over)) {
            status = PYST_TRAJ_OVERFLOW;
            break;
          }
          if (!__any_sync(0xffffffffu, neg)) {
            ok = true;
            break;
          }
          tau = __dmul_rn(tau, 0.5);
          retry++;
          if (retry > ra.max_leap_retries) {
            status = PYST_TRAJ_LEAP_RETRY;
            break;
          }
        }
        if (!ok) break;
        leap_q++;
        const double tn = __dadd_rn(t, tau);
        // firing count and hash (lane 0 walks K in order)
        int64_t fired = 0;
        for (int j = j0; j < j1; ++j) {
          fired += ws.K[j];
          if (SCORE) {
            score_acc[j] = __dadd_rn(score_acc[j], (double)ws.K[j]);
          }
        }
        if (SCORE) {
          for (int j = j0; j < j1; ++j) {
            // integral term kept in a separate pass of the same slot
            score_acc[R + j] =
                __dadd_rn(score_acc[R + j], __dmul_rn((double)ws.a[j], tau));
          }
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1)
          fired += __shfl_xor_sync(0xffffffffu, fired, d);
        if (lane == 0) {
          h = seq_mix(h, PYST_LEAP_TAG);
          for (int j = 0; j < R; ++j)
            if (ws.K[j] != 0)
              h = seq_mix(h, ((uint64_t)j << 32) | (uint32_t)ws.K[j]);
        }
        bool done = false;
        while (tn >= m.time(f)) {
          const double frac = __ddiv_rn(__dsub_rn(m.time(f), t), tau);
          for (int k = lane; k < kappa; k += 32) {
            const int i = m.out(k);
            const double inc = rint(__dmul_rn((double)ws.slot[i], frac));
            store_sample(o, ita, k, f, ws.x[i] + (int)inc);
          }
          f++;
          if (f == ita) {
            done = true;
            break;
          }
        }
        __syncwarp();
        for (int i = lane; i < S; i += 32)
          ws.x[i] = (int)((int64_t)ws.x[i] + ws.slot[i]);
        __syncwarp();
        events += fired;
        t = tn;
        if (done) break;
        continue;
      }
    }
    // ------------------------ one direct-method step -------------------
    steps++;
    const uint4 w = next_block(rs);
    const double tau = __ddiv_rn(-pyst_log(u53(w.x, w.y)), a0);
    const double r = __dmul_rn(u53(w.z, w.w), a0);
    const int sel = warp_select(ws.a, part, incl, r, j0, j1, lane, nullptr);
    const double tn = __dadd_rn(t, tau);
    if (SCORE) {
      const double dt = (tn >= t_end) ? __dsub_rn(t_end, t) : tau;
      for (int j = j0; j < j1; ++j)
        score_acc[R + j] =
            __dadd_rn(score_acc[R + j], __dmul_rn((double)ws.a[j], dt));
    }
    bool done = false;
    while (tn >= m.time(f)) {
      for (int k = lane; k < kappa; k += 32)
        store_sample(o, ita, k, f, ws.x[m.out(k)]);
      f++;
      if (f == ita) {
        done = true;
        break;
      }
    }
    t = tn;
    if (done) break;
    bool over = false;
    if (lane == 0) {
      const int e1 = m.netptr(sel + 1);
      for (int e = m.netptr(sel); e < e1; ++e) {
        const uint32_t ne = m.net(e);
        const int sp = ent_lo(ne);
        const int64_t nx = (int64_t)ws.x[sp] + ent_hi_s16(ne);
        if (nx < 0 || nx > PYST_I32MAX) over = true;
        else ws.x[sp] = (int)nx;
      }
      if (SCORE) score_acc[sel] = __dadd_rn(score_acc[sel], 1.0);
    }
    __syncwarp();
    if (__any_sync(0xffffffffu, over)) {
      status = PYST_TRAJ_OVERFLOW;
      break;
    }
    events++;
    h = seq_mix(h, (uint64_t)sel);
    if (TAU) {
      if (--ssa_left <= 0) ssa_mode = false;
    }
  }
  __syncwarp();
  for (; f < ita; ++f)
    for (int k = lane; k < kappa; k += 32)
      store_sample(o, ita, k, f, fill_state ? ws.x[m.out(k)] : -1);
  if (lane == 0) {
    if (o.status) *o.status = (uint8_t)status;
    if (o.events) *o.events = events;
    if (o.seqhash) *o.seqhash = h;
    if (o.t_final) *o.t_final = t;
  }
  if (SCORE && o.score) {
    __syncwarp();
    for (int j = lane; j < R; j += 32)
      o.score[j] = __dsub_rn(score_acc[j], score_acc[R + j]);
  }
  __syncwarp();
}

}  // namespace pyst
