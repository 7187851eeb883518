// One-trajectory-per-thread kernel for a single model (the plain form):
// replaces kernel_Gillespie (mod/simulator/cuGillespie/gillespie.py:27-149)
// and the kernel_P1_P2 / kernel_P3 pair with its host round loop
// (mod/simulator/cuTauLeaping/cuTauLeaping.py:49-76).  Built once per
// (PYST_TAU, PYST_SCORE) flavour.
#include "pyst_launch.cuh"

#ifndef PYST_TAU
#error "PYST_TAU must be defined"
#endif
#ifndef PYST_SCORE
#error "PYST_SCORE must be defined"
#endif

namespace pyst {
// nvcc gives template functions of an anonymous namespace weak external
// linkage on the host side, so the flavours built from this file would be
// merged at link time; a per-flavour namespace keeps them apart.
namespace PYST_CAT(thread_flavour_, PYST_TAU, PYST_SCORE) {

// Blocks of 128 threads per SM the register allocation must allow: 6
// (at most 80 registers) measured fastest for the throughput-bound
// telegraph gradient workload (1M trajectories: 221 ms, against 226 at 5,
// 230 with no bound) and costs the latency-bound 1024-trajectory
// Lotka-Volterra run under 1%; 8 (64 registers) spills (339 vs 289 ms).
#ifndef PYST_THREAD_MINB
#define PYST_THREAD_MINB 6
#endif



// PK: kPkPacked for models whose every reaction packs (the host checks),
// kPkLists otherwise (general kinetic laws included).  RX: MAXR when the
// model has exactly MAXR reactions (the host checks), else 0.
template <int MAXR, bool TAU, bool SCORE, int PK, int RX = 0>
__global__ void __launch_bounds__(128, PYST_THREAD_MINB)
    k_plain_thread(const uint32_t* __restrict__ gblob, int blob_words,
                   int64_t n_traj, uint64_t id_base, RunArgs ra, OutBase ob,
                   unsigned long long* queue) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* sblob = (uint32_t*)smem;
  uint64_t* bar = (uint64_t*)(smem + (size_t)blob_words * 4);
  // packed reaction descriptors (register-array engine only), then the
  // species columns
  const int R = (int)__ldg(gblob + PYST_H_R);
  uint32_t* pk = (uint32_t*)(smem + (size_t)blob_words * 4 + 16);
  int32_t* xbase =
      (int32_t*)((unsigned char*)pk + (MAXR > 0 ? packed_bytes(R) : 0));
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const bool ok = stage_blob(sblob, gblob, blob_words, bar, 0,
                             ra.stage_polls);
  const int bs = blockDim.x;
  const int64_t nthreads = (int64_t)gridDim.x * bs;
  // first trajectory by thread index, later ones from the shared queue, so
  // a thread whose trajectory ends early takes the next unstarted one
  int64_t u = blockIdx.x * (int64_t)bs + threadIdx.x;
  if (!ok) {
    mbar_drain(bar, 0);  // let a late copy land before the block exits
    while (u < n_traj) {
      mark_staging_failure(ob, u);
      u = nthreads + (int64_t)atomicAdd(queue, 1ull);
    }
    return;
  }
  ModelView m;
  m.load(sblob);
  if (MAXR > 0) {
    m.pk = pk;
    m.fast = __syncthreads_and(pack_reactions(m, pk)) != 0;
  }
  int32_t* xcol = xbase + threadIdx.x;
  int64_t* slot = (int64_t*)(xbase + (size_t)m.S * bs) + threadIdx.x;
  while (u < n_traj) {
    const TrajOut o = ob.at(0, u, 0, 0, ob.stride, m.R);
    if constexpr (MAXR == 0)
      run_thread_big<TAU>(m, xcol, slot, bs, ra, id_base + (uint64_t)u, o);
    else
      run_thread<MAXR, TAU, SCORE, PK, RX>(m, xcol, slot, bs, ra,
                                       id_base + (uint64_t)u, o);
    u = nthreads + (int64_t)atomicAdd(queue, 1ull);
  }
}

// ---------------------------------------------------------------------
// Species counts in registers (at most MAXS), read and written by
// unrolled selects: the lane tree's state.  (A one-thread-per-trajectory
// direct-method kernel with species in registers measured slower than the
// shared-memory columns of k_plain_thread: telegraph, 1M trajectories,
// 175 vs 165 ms -- the selects cost more than the load they replace.)
template <int MAXS>
__device__ __forceinline__ int reg_get(const int (&x)[MAXS], int sp) {
  int v = x[0];
#pragma unroll
  for (int s = 1; s < MAXS; ++s) v = (sp == s) ? x[s] : v;
  return v;
}

// x += the packed net change d, entry by entry with the range check of
// thread_round (an entry that would leave [0, 2^31) is skipped and flags
// the step); false if any entry was out of range.
template <int MAXS>
__device__ __forceinline__ bool reg_apply(int (&x)[MAXS], uint32_t d) {
  bool ok = true;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    if (q < pnet_count(d)) {
      const int sp = pnet_species(d, q);
      const int64_t nx = (int64_t)reg_get(x, sp) + pnet_delta(d, q);
      if (nx < 0 || nx > PYST_I32MAX) {
        ok = false;
      } else {
#pragma unroll
        for (int s = 0; s < MAXS; ++s)
          if (s == sp) x[s] = (int)nx;
      }
    }
  }
  return ok;
}

// The direct-method selection for uniform-times-total r, as thread_round.
template <int MAXR>
__device__ __forceinline__ int select_reaction(const float (&a)[MAXR], int R,
                                               double r) {
  double cum = 0.0;
  int lastnz = -1, sel = -1;
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
  return sel < 0 ? lastnz : sel;
}

// Exponential variate and uniform of main-stream block `blk`.
__device__ __forceinline__ void step_variates(Stream& rs, uint64_t blk,
                                              double& e, double& u) {
  rs.n = blk;
  const uint4 w = next_block(rs);
  e = -pyst_log(u53(w.x, w.y));
  u = u53(w.z, w.w);
}

#if !PYST_TAU && !PYST_SCORE
// Lane groups for runs too small to fill the GPU (direct method): each
// trajectory is a long dependent chain of steps, so with at most a few
// warps per SM the step latency, not issue throughput, sets the time.
// kGroupLanes lanes share one trajectory (thread_round's LG form), which
// takes the Philox and log work of the other steps off each step's chain.
// Trajectory u is group u (static assignment); lane 0 of a group writes.
// A whole warp per trajectory measured fastest (Lotka-Volterra, 1024
// trajectories: 206.7 ms at 32 lanes, 217.1 at 16, 236.1 at 8): the warp
// then never diverges between trajectories.
#ifndef PYST_GROUP_LANES
#define PYST_GROUP_LANES 32
#endif
constexpr int kGroupLanes = PYST_GROUP_LANES;
// 0 keeps the lane groups on the plain lockstep loop (no lane tree)
#ifndef PYST_SPEC_TREE
#define PYST_SPEC_TREE 1
#endif
// runs of at most this many trajectories per SM take the lane groups
constexpr int kGroupMaxPerSm = 16;

// ---------------------------------------------------------------------
// Speculative lane tree (the lane groups' fast path for small mass-action
// models).  A step's selection j depends on the state, which depends on the
// previous selection: one dependent chain per trajectory.  Here the 32
// lanes of the trajectory's warp evaluate the next D steps at once: the
// lane at depth d with path (j_1 .. j_d) takes the state after firing
// j_1 .. j_d, computes its propensities, total, tau and selection for step
// d + 1 (with step d + 1's random numbers), and a few ballots publish every
// lane's selection, so each lane walks the tree from the root along the
// selections to the true path.  Lanes per depth grow as R^d, so the full
// depth D is 5 for R <= 2 (31 lanes), 3 for R <= 4 (21) and 2 for R <= 8
// (9); the lanes left over cover part of level D, so a pass whose true
// path is there takes one step more: Lotka-Volterra (R = 3) advances 3
// steps per pass on 13 lanes, or 4 when its path is among the 19 of 27
// covered at level 3.
// The passes commit only when none of the D steps reaches a sample time,
// absorbs, runs out of step budget or leaves the int32 range; otherwise D
// exact single steps run instead (thread_round's order of operations, which
// handles every such case).  Every lane does exactly the arithmetic of the
// step it evaluates, so results are those of one thread per trajectory,
// bit for bit.  Species counts (at most MAXS) live in registers, read and
// written by unrolled selects.
// Lanes of a D-level tree for R reactions: 1 + R + ... + R^(D-1).
__host__ __device__ constexpr int spec_lanes(int R, int D) {
  return D <= 0 ? 0 : 1 + R * spec_lanes(R, D - 1);
}

// One whole trajectory by the calling warp (all 32 lanes; lane 0 writes).
// D levels (compile time; the caller checks spec_lanes(R, D) <= 32), at
// most MAXS species in registers; RX: the model's reaction count when the
// caller fixes it at compile time, else 0.
template <int MAXR, int MAXS, int D, int RX>
__device__ void run_spec_tree(const ModelView& m, const RunArgs& ra,
                              uint64_t traj_id, const TrajOut& o) {
  const int R = RX ? RX : m.R, S = m.S, ita = m.ita, kappa = m.kappa;
  const int lane = threadIdx.x & 31;
  // this lane's depth dl and path j_1 .. j_dl (base-R digits of its index
  // within the depth, first firing first)
  // Full levels 0 .. D-1 take `used` lanes; the remaining lanes cover the
  // first `extra` paths of level D, so a pass whose true path is among
  // them commits D + 1 steps.
  const int used = spec_lanes(R, D);
  int width_d = 1;
  for (int d = 0; d < D; ++d) width_d *= R;
  const int extra = 32 - used < width_d ? 32 - used : width_d;
  int dl = 0, il = 0;
  {
    int st = 0, w = 1;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      if (lane >= st && lane < st + w) {
        dl = d;
        il = lane - st;
      }
      st += w;
      w *= R;
    }
    if (lane >= used && lane < used + extra) {
      dl = D;
      il = lane - used;
    }
  }
  const bool in_tree = lane < used + extra;
  // the path's net change, and the extremes of its running sum, per species
  // (the states along the path stay in [0, 2^31) iff x + lo >= 0 and
  // x + hi < 2^31), fixed for the whole trajectory
  int dx[MAXS], lo[MAXS], hi[MAXS];
#pragma unroll
  for (int s = 0; s < MAXS; ++s) dx[s] = lo[s] = hi[s] = 0;
  {
    int pw = 1;
    for (int k = 1; k < dl; ++k) pw *= R;
    for (int k = 0; k < dl; ++k) {
      const int j = (il / pw) % R;
      pw = pw > 1 ? pw / R : 1;
      const uint32_t d = m.pk[R + j];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        if (q < pnet_count(d)) {
          const int sp = pnet_species(d, q);
#pragma unroll
          for (int s = 0; s < MAXS; ++s) {
            if (s == sp) {
              dx[s] += pnet_delta(d, q);
              lo[s] = dx[s] < lo[s] ? dx[s] : lo[s];
              hi[s] = dx[s] > hi[s] ? dx[s] : hi[s];
            }
          }
        }
      }
    }
  }

  // the reactions' rates and packed descriptors, in registers for the
  // whole trajectory
  float rate[MAXR];
  uint32_t fac[MAXR], net[MAXR];
#pragma unroll
  for (int j = 0; j < MAXR; ++j) {
    rate[j] = j < R ? m.rate(j) : 0.0f;
    fac[j] = j < R ? m.pk[j] : 0u;
    net[j] = j < R ? m.pk[R + j] : 0u;
  }
  // propensities (FP32, packed descriptors) and their FP64 total, with
  // thread_round's operations in its order
  auto props = [&](const int (&xx)[MAXS], float (&a)[MAXR]) {
    double a0 = 0.0;
    auto xget = [&](int i) { return reg_get(xx, i); };
#pragma unroll
    for (int j = 0; j < MAXR; ++j) {
      if (j >= R) break;
      a[j] = propensity_packed(rate[j], fac[j], xget);
      a0 = __dadd_rn(a0, (double)a[j]);
    }
    return a0;
  };
  // net change of reaction sel (of reaction 0 for sel < 0)
  auto net_of = [&](int sel) {
    uint32_t d = net[0];
#pragma unroll
    for (int j = 1; j < MAXR; ++j) d = sel == j ? net[j] : d;
    return d;
  };
  // the firing-sequence hash only when the caller asked for it
  const bool want_h = o.seqhash != nullptr;

  Stream rs = make_stream(ra.seed, traj_id);
  int x[MAXS];
#pragma unroll
  for (int s = 0; s < MAXS; ++s) x[s] = s < S ? m.x0(s) : 0;
  // step variates: lane g holds blocks vb + g (cur) and vb + 32 + g (nxt).
  // A pass reads the steps base .. base + D of vb + 32 offsets, base =
  // steps - vb < 32: offset g (g >= base) from cur of lane g, offset 32 + g
  // (g < base) from nxt of lane g, so each lane offers the one it owns in
  // the window (e_w, u_w) and a read is one shuffle.
  uint64_t vb = 0;
  double e_c, u_c, e_n, u_n, e_w, u_w;
  step_variates(rs, (uint64_t)lane, e_c, u_c);
  step_variates(rs, 32u + (uint64_t)lane, e_n, u_n);
  auto variate = [&](int64_t step, double& e, double& u) {
    const int own = (int)(step - (int64_t)vb) & 31;
    e = __shfl_sync(0xffffffffu, e_w, own);
    u = __shfl_sync(0xffffffffu, u_w, own);
  };

  double t = 0.0;
  int f = 0;
  double tf = m.time(0);
  int64_t steps = 0, events = 0;
  uint64_t h = PYST_FNV_OFFSET;
  int status = PYST_TRAJ_DONE;
  bool fill_state = false, done = false;
  const int64_t budget = ra.step_budget;
  constexpr int kSelBits = MAXR <= 2 ? 1 : (MAXR <= 4 ? 2 : 3);

  while (!done) {
    if (steps - (int64_t)vb >= 32) {
      vb += 32;
      e_c = e_n;
      u_c = u_n;
      step_variates(rs, vb + 32u + (uint64_t)lane, e_n, u_n);
    }
    {
      const bool in_cur = lane >= (int)(steps - (int64_t)vb);
      e_w = in_cur ? e_c : e_n;
      u_w = in_cur ? u_c : u_n;
    }
    bool committed = false;
    if (D > 1 && steps + D <= budget) {
      // ---- every lane: the step at the end of its path --------------
      int xs[MAXS];
      bool ok = in_tree;
#pragma unroll
      for (int s = 0; s < MAXS; ++s) {
        xs[s] = x[s] + dx[s];
        ok &= x[s] + lo[s] >= 0 && x[s] <= (int)PYST_I32MAX - hi[s];
      }
      float a[MAXR];
      const double a0 = props(xs, a);
      double e, u;
      variate(steps + dl, e, u);
      const double tau = __ddiv_rn(e, a0);
      const int sel = select_reaction<MAXR>(a, R, __dmul_rn(u, a0));
      ok &= a0 != 0.0;
      // the state after this lane's step (needed from the deepest lane of
      // the true path, at level D - 1 or D): its range check joins the
      // lane's flag
      if (dl >= D - 1) ok &= reg_apply(xs, net_of(sel));
      unsigned sb[kSelBits];
#pragma unroll
      for (int b = 0; b < kSelBits; ++b)
        sb[b] = __ballot_sync(0xffffffffu, (sel >> b) & 1);
      const unsigned bad = __ballot_sync(0xffffffffu, !ok);
      // ---- walk the tree along the selections (uniform) ---------------
      int J[D + 1], L[D + 1];
      unsigned badpath = 0u;
      int dn = D;  // steps this pass commits
      {
        int i = 0, st = 0, w = 1;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          const int ln = st + i;
          badpath |= (bad >> ln) & 1u;
          int j = 0;
#pragma unroll
          for (int b = 0; b < kSelBits; ++b)
            j |= (int)((sb[b] >> ln) & 1u) << b;
          J[d] = j;
          L[d] = ln;
          i = i * R + j;
          st += w;
          w *= R;
        }
        // one step more when the partial level holds the path, its step
        // is sound and within the budget (otherwise the next pass or the
        // exact steps take it)
        const int ln = used + i;
        L[D] = ln;
        J[D] = 0;
        if (i < extra && !((bad >> ln) & 1u) && steps + D + 1 <= budget) {
          int j = 0;
#pragma unroll
          for (int b = 0; b < kSelBits; ++b)
            j |= (int)((sb[b] >> ln) & 1u) << b;
          J[D] = j;
          dn = D + 1;
        }
      }
      if (!badpath) {
        double tt = t;
#pragma unroll
        for (int d = 0; d <= D; ++d) {
          const double td = __shfl_sync(0xffffffffu, tau, L[d]);
          if (d < dn) tt = __dadd_rn(tt, td);
        }
        if (tt < tf) {
          const int last = dn > D ? L[D] : L[D - 1];
#pragma unroll
          for (int s = 0; s < MAXS; ++s)
            x[s] = __shfl_sync(0xffffffffu, xs[s], last);
          if (want_h) {
#pragma unroll
            for (int d = 0; d <= D; ++d)
              if (d < dn) h = seq_mix(h, (uint64_t)J[d]);
          }
          t = tt;
          steps += dn;
          events += dn;
          committed = true;
        }
      }
    }
    if (committed) continue;
    // ---- D exact single steps ------------------------------------------
    for (int q = 0; q < D && !done; ++q) {
      float a[MAXR];
      const double a0 = props(x, a);
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
      double e, u;
      variate(steps, e, u);
      steps++;
      const double tau = __ddiv_rn(e, a0);
      const int sel = select_reaction<MAXR>(a, R, __dmul_rn(u, a0));
      const double tn = __dadd_rn(t, tau);
      while (tn >= tf) {
        if (lane == 0)
          for (int k = 0; k < kappa; ++k)
            store_sample(o, ita, k, f, reg_get(x, m.out(k)));
        f++;
        if (f == ita) {
          done = true;
          break;
        }
        tf = m.time(f);
      }
      t = tn;
      if (done) break;
      if (!reg_apply(x, net_of(sel))) {
        status = PYST_TRAJ_OVERFLOW;
        done = true;
        break;
      }
      events++;
      if (want_h) h = seq_mix(h, (uint64_t)sel);
    }
  }
  if (lane == 0) {
    for (; f < ita; ++f)
      for (int k = 0; k < kappa; ++k)
        store_sample(o, ita, k, f,
                     fill_state ? reg_get(x, m.out(k)) : -1);
    if (o.status) *o.status = (uint8_t)status;
    if (o.events) *o.events = events;
    if (o.seqhash) *o.seqhash = h;
    if (o.t_final) *o.t_final = t;
  }
}

// species held in registers by the lane tree
constexpr int kSpecMaxSpecies = 8;

// One warp per trajectory, the lane tree (D levels, at most MAXS species);
// launched only for models whose every reaction packs
// (blob_reaction_packable) with at most MAXS species.  4 blocks of 128
// threads per SM: a run of 148 x 16 trajectories is resident at once.
template <int MAXR, int MAXS, int D, int RX>
__global__ void __launch_bounds__(128, 4)
    k_plain_tree(const uint32_t* __restrict__ gblob, int blob_words,
                 int64_t n_traj, uint64_t id_base, RunArgs ra, OutBase ob) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* sblob = (uint32_t*)smem;
  uint64_t* bar = (uint64_t*)(smem + (size_t)blob_words * 4);
  uint32_t* pk = (uint32_t*)(smem + (size_t)blob_words * 4 + 16);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const bool ok = stage_blob(sblob, gblob, blob_words, bar, 0,
                             ra.stage_polls);
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const bool leader = (threadIdx.x & 31) == 0;
  int64_t u = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (!ok) {
    mbar_drain(bar, 0);  // let a late copy land before the block exits
    for (; u < n_traj; u += nwarps)
      if (leader) mark_staging_failure(ob, u);
    return;
  }
  ModelView m;
  m.load(sblob);
  m.pk = pk;
  // the host launches this kernel only when every reaction packs, and the
  // device packer decides with the same predicate
  m.fast = __syncthreads_and(pack_reactions(m, pk)) != 0;
  for (; u < n_traj; u += nwarps) {
    const TrajOut o = ob.at(0, u, 0, 0, ob.stride, m.R);
    run_spec_tree<MAXR, MAXS, D, RX>(m, ra, id_base + (uint64_t)u, o);
  }
}

template <int MAXR, int MAXS, int D, int RX>
int launch_tree(const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
                uint64_t id_base, const RunArgs& ra, const OutBase& ob,
                cudaStream_t st) {
  auto kf = k_plain_tree<MAXR, MAXS, D, RX>;
  const size_t smem = (size_t)mi.words * 4 + 16 + packed_bytes(mi.R);
  const int rc = set_smem(kf, smem);
  if (rc) return rc;
  const int bs = 128;
  const int64_t grid = (n * 32 + bs - 1) / bs;
  kf<<<(unsigned)grid, bs, smem, st>>>(d_blob, mi.words, n, id_base, ra, ob);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

// The lane tree for a packable model of at most 8 reactions and
// kSpecMaxSpecies species: depth 5 for R <= 2, 3 for R <= 4, 2 for R <= 8;
// the reaction count fixed at compile time for R = 2, 3, 4, the species
// registers sized 2, 4 or 8.
template <int MAXS>
int launch_tree_s(const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
                  uint64_t id_base, const RunArgs& ra, const OutBase& ob,
                  cudaStream_t st) {
  switch (mi.R) {
    case 2:
      return launch_tree<2, MAXS, 5, 2>(d_blob, mi, n, id_base, ra, ob, st);
    case 3:
      return launch_tree<3, MAXS, 3, 3>(d_blob, mi, n, id_base, ra, ob, st);
    case 4:
      return launch_tree<4, MAXS, 3, 4>(d_blob, mi, n, id_base, ra, ob, st);
    default:
      return mi.R < 2
                 ? launch_tree<2, MAXS, 5, 0>(d_blob, mi, n, id_base, ra, ob,
                                              st)
                 : launch_tree<8, MAXS, 2, 0>(d_blob, mi, n, id_base, ra, ob,
                                              st);
  }
}

int launch_tree_for(const uint32_t* d_blob, const HostModelInfo& mi,
                    int64_t n, uint64_t id_base, const RunArgs& ra,
                    const OutBase& ob, cudaStream_t st) {
  if (mi.S <= 2)
    return launch_tree_s<2>(d_blob, mi, n, id_base, ra, ob, st);
  if (mi.S <= 4)
    return launch_tree_s<4>(d_blob, mi, n, id_base, ra, ob, st);
  return launch_tree_s<8>(d_blob, mi, n, id_base, ra, ob, st);
}

template <int MAXR, int LG>
__global__ void __launch_bounds__(128)
    k_plain_group(const uint32_t* __restrict__ gblob, int blob_words,
                  int64_t n_traj, uint64_t id_base, RunArgs ra, OutBase ob) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* sblob = (uint32_t*)smem;
  uint64_t* bar = (uint64_t*)(smem + (size_t)blob_words * 4);
  const int R = (int)__ldg(gblob + PYST_H_R);
  uint32_t* pk = (uint32_t*)(smem + (size_t)blob_words * 4 + 16);
  int32_t* xbase = (int32_t*)((unsigned char*)pk + packed_bytes(R));
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const bool ok = stage_blob(sblob, gblob, blob_words, bar, 0,
                             ra.stage_polls);
  const int bs = blockDim.x;
  const int64_t ngroups = (int64_t)gridDim.x * bs / LG;
  const bool leader = (threadIdx.x & (LG - 1)) == 0;
  int64_t u = (blockIdx.x * (int64_t)bs + threadIdx.x) / LG;
  if (!ok) {
    mbar_drain(bar, 0);  // let a late copy land before the block exits
    for (; u < n_traj; u += ngroups)
      if (leader) mark_staging_failure(ob, u);
    return;
  }
  ModelView m;
  m.load(sblob);
  m.pk = pk;
  m.fast = __syncthreads_and(pack_reactions(m, pk)) != 0;
  int32_t* xcol = xbase + threadIdx.x;
  int64_t* slot = (int64_t*)(xbase + (size_t)m.S * bs) + threadIdx.x;
  for (; u < n_traj; u += ngroups) {
    const TrajOut o = ob.at(0, u, 0, 0, ob.stride, m.R);
    const uint64_t id = id_base + (uint64_t)u;
    TState st;
    thread_init<false>(m, xcol, bs, st);
    double integ[1] = {0.0};
    int cnt[1] = {0};
    if (m.fast)
      thread_round<MAXR, false, false, kPkPacked, LG>(
          m, xcol, slot, bs, bs, ra, id, st, integ, cnt, o, 0x7fffffff,
          0x7fffffff, false);
    else
      thread_round<MAXR, false, false, kPkLists, LG>(
          m, xcol, slot, bs, bs, ra, id, st, integ, cnt, o, 0x7fffffff,
          0x7fffffff, false);
    if (leader) thread_finish<MAXR, false>(m, xcol, bs, st, integ, cnt, o);
  }
}

template <int MR>
int launch_group(const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
                 uint64_t id_base, const RunArgs& ra, const OutBase& ob,
                 int bs, cudaStream_t st, size_t smem) {
  auto kf = k_plain_group<MR, kGroupLanes>;
  const int rc = set_smem(kf, smem);
  if (rc) return rc;
  const int64_t grid = (n * kGroupLanes + bs - 1) / bs;
  kf<<<(unsigned)grid, bs, smem, st>>>(d_blob, mi.words, n, id_base, ra, ob);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}
#endif

template <class K>
int launch_k(K kf, const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
             uint64_t id_base, const RunArgs& ra, const OutBase& ob, int bs,
             cudaStream_t st, size_t smem, unsigned long long* queue) {
  const int rc = set_smem(kf, smem);
  if (rc) return rc;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf, bs, smem);
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (n + bs - 1) / bs;
  const int64_t cap = (int64_t)num_sms() * per_sm;
  if (grid > cap) grid = cap;
  kf<<<(unsigned)grid, bs, smem, st>>>(d_blob, mi.words, n, id_base, ra, ob,
                                       queue);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

template <int MR>
int launch_one(const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
               uint64_t id_base, const RunArgs& ra, const OutBase& ob, int bs,
               cudaStream_t st, size_t smem, unsigned long long* queue) {
  // the packed-descriptor form compiled on its own for packable models
  auto kf = (MR > 0 && mi.packable)
                ? k_plain_thread<MR, (bool)PYST_TAU, (bool)PYST_SCORE,
                                 kPkPacked>
                : k_plain_thread<MR, (bool)PYST_TAU, (bool)PYST_SCORE,
                                 kPkLists>;
  return launch_k(kf, d_blob, mi, n, id_base, ra, ob, bs, st, smem, queue);
}

// A packable model of 2 to 8 reactions: the packed form with the reaction
// count fixed at compile time (its per-reaction loops carry no run-time
// bound): telegraph gradient forward, 1M trajectories, 208.5 -> 173.6 ms;
// Schlogl direct method, 262144 trajectories, 170 -> 152.5 ms.
template <int RXV>
int launch_exact(const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
                 uint64_t id_base, const RunArgs& ra, const OutBase& ob,
                 int bs, cudaStream_t st, size_t smem,
                 unsigned long long* queue) {
  return launch_k(
      k_plain_thread<RXV, (bool)PYST_TAU, (bool)PYST_SCORE, kPkPacked, RXV>,
      d_blob, mi, n, id_base, ra, ob, bs, st, smem, queue);
}

int launch_exact_r(const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
                   uint64_t id_base, const RunArgs& ra, const OutBase& ob,
                   int bs, cudaStream_t st, size_t smem,
                   unsigned long long* queue) {
  switch (mi.R) {
#define PYST_EXACT_CASE(r)                                                  \
  case r:                                                                   \
    return launch_exact<r>(d_blob, mi, n, id_base, ra, ob, bs, st, smem,    \
                           queue);
    PYST_EXACT_CASE(2)
    PYST_EXACT_CASE(3)
    PYST_EXACT_CASE(4)
    PYST_EXACT_CASE(5)
    PYST_EXACT_CASE(6)
    PYST_EXACT_CASE(7)
    PYST_EXACT_CASE(8)
#undef PYST_EXACT_CASE
    default:
      return PYST_EUNSUPPORTED;
  }
}

}  // namespace (flavour)
using namespace PYST_CAT(thread_flavour_, PYST_TAU, PYST_SCORE);

int PYST_CAT(launch_plain_thread_, PYST_TAU, PYST_SCORE)(
    int maxr, const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
    uint64_t id_base, const RunArgs& ra, const OutBase& ob, int bs,
    unsigned long long* queue, cudaStream_t st) {
  const size_t smem =
      (size_t)mi.words * 4 + 16 +
      (maxr <= PYST_THREAD_MAX_REACTIONS ? packed_bytes(mi.R) : 0) +
      (size_t)bs * mi.S * (PYST_TAU ? 12 : 4);
  if (smem > kMaxDynSmem) return PYST_EUNSUPPORTED;
  if (n <= 0) return PYST_OK;
  if (cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st) !=
      cudaSuccess)
    return PYST_ECUDA;
#if !PYST_SCORE
  if (maxr > PYST_THREAD_MAX_REACTIONS)
    return launch_one<0>(d_blob, mi, n, id_base, ra, ob, bs, st, smem, queue);
#else
  if (maxr > PYST_THREAD_MAX_REACTIONS) return PYST_EUNSUPPORTED;
#endif
#if !PYST_TAU && !PYST_SCORE
  // runs too small to fill the GPU: at most kGroupMaxPerSm trajectories per
  // SM, each on a whole warp (kGroupLanes = 32 lanes by default) -- the
  // lane tree for packable models of at most kSpecMaxSpecies species, the
  // lockstep lane groups otherwise
  if (maxr <= 8 && bs <= 128 && bs % kGroupLanes == 0 &&
      n <= (int64_t)num_sms() * kGroupMaxPerSm) {
    if (PYST_SPEC_TREE && mi.packable && mi.S <= kSpecMaxSpecies)
      return launch_tree_for(d_blob, mi, n, id_base, ra, ob, st);
    if (maxr <= 4)
      return launch_group<4>(d_blob, mi, n, id_base, ra, ob, bs, st, smem);
    return launch_group<8>(d_blob, mi, n, id_base, ra, ob, bs, st, smem);
  }
#endif
  if (mi.packable && mi.R >= 2 && mi.R <= 8)
    return launch_exact_r(d_blob, mi, n, id_base, ra, ob, bs, st, smem,
                          queue);
  if (maxr <= 4)
    return launch_one<4>(d_blob, mi, n, id_base, ra, ob, bs, st, smem, queue);
  if (maxr <= 8)
    return launch_one<8>(d_blob, mi, n, id_base, ra, ob, bs, st, smem, queue);
  if (maxr <= 16)
    return launch_one<16>(d_blob, mi, n, id_base, ra, ob, bs, st, smem,
                          queue);
  return launch_one<32>(d_blob, mi, n, id_base, ra, ob, bs, st, smem, queue);
}

}  // namespace pyst
