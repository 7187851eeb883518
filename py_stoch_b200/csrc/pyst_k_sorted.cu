// Mode-sorted persistent kernel for thread-mapped tau-leaping.
//
// In tau-leaping each trajectory is, at any time, either in an SSA
// fallback round (mod/simulator/cuTauLeaping/P3.py:71-151) or leaping
// (P1_P2.py:96-297).  The reference runs the two as separate kernels, so in
// each launch the threads of the other mode sit idle.  Here a block keeps a
// pool of (up to 2) x blockDim trajectory slots in shared memory (species
// counts and the per-trajectory state between rounds) and runs in rounds: it
// counting-sorts the occupied slots by mode, picks up to blockDim of them --
// whole warps of one mode where it can, rotating through each mode's slots
// so that every trajectory keeps advancing -- and each thread advances the
// trajectory in its picked slot for up to cap_ssa SSA steps or cap_leap
// leaps (stopping early when a DECIDE switches mode).  A finished
// trajectory's slot is refilled from the global work queue.  With more slots
// than threads every trajectory of a launch that fits the pools starts at
// once, so no long trajectory starts late, and the mode mix of a round can
// be chosen from a larger set.  Per-trajectory arithmetic is exactly that of
// run_thread, so results do not depend on the schedule.  Built once per
// PYST_SCORE flavour.
#include "pyst_launch.cuh"

namespace pyst {
// see pyst_k_thread.cu: per-flavour namespace, not an anonymous one
namespace PYST_CAT(sorted_flavour_, PYST_SCORE, ) {

constexpr bool kScore = (bool)PYST_SCORE;
// Largest block (threads) and the register budget: one block of
// PYST_SORTED_MAX_BLOCK threads per SM.  896 threads leave 72 registers
// each and measured 4% faster on the Schlogl workload than 1024 threads at
// 64 registers (register spills) and than 768 (fewer warps); the score
// flavour keeps 128-thread blocks with 4 resident (its accumulators need
// the registers).
#ifndef PYST_SORTED_MAX_BLOCK
#define PYST_SORTED_MAX_BLOCK 896
#endif
constexpr int kMaxBlock = kScore ? 128 : PYST_SORTED_MAX_BLOCK;
constexpr int kMinBlocks = kScore ? 4 : 1;
// Preferred block size: the launcher takes the largest size up to this
// whose shared memory fits, first with PYST_SORTED_POOL slots per thread,
// then with one.
#ifndef PYST_SORTED_BLOCK
#define PYST_SORTED_BLOCK PYST_SORTED_MAX_BLOCK
#endif
#ifndef PYST_SORTED_POOL
#define PYST_SORTED_POOL 2
#endif
// The one warp per round that holds both SSA and leaping slots runs rounds
// of half length.
#ifndef PYST_MIXED_HALF
#define PYST_MIXED_HALF 1
#endif
constexpr int kMaxPool = PYST_SORTED_POOL;
static_assert(kMaxPool <= 2,
              "the schedule's scan holds at most 64 slot groups");
constexpr int kPrefBlock =
    PYST_SORTED_BLOCK < kMaxBlock ? PYST_SORTED_BLOCK : kMaxBlock;

struct SortedSmem {
  uint32_t* blob;
  uint64_t* bar;
  uint32_t* pk;      // [2 * maxr] packed reaction descriptors
  int64_t* scratch;  // [S][block] leap scratch of the running threads
  double* t;         // per slot [pool * block] ...
  uint64_t* n;
  int64_t* events;
  int64_t* steps;
  uint64_t* h;
  int64_t* traj;     // trajectory index, -1 for an empty slot
  double* integ;     // [MAXR][slots]
  int32_t* x;        // [S][slots] species counts
  int32_t* f;
  uint32_t* leap_q;
  int32_t* ssa_left;
  int32_t* flags;
  int32_t* cnt;      // [MAXR][slots]
  int32_t* run;      // [block] slot run by each thread this round
  int32_t* gcnt;     // [2][pool * block / 32] SSA / leaping slots per group
  int slots;         // pool * block: the stride of every per-slot array
};

__host__ __device__ inline size_t sorted_smem_bytes(int blob_words, int S,
                                                    int maxr, int pool,
                                                    int block) {
  const size_t slots = (size_t)pool * block;
  size_t b = (size_t)blob_words * 4 + 16 + packed_bytes(maxr);
  b += (size_t)S * block * 8;
  b += slots * (8 * 6 + 4 * 4);
  b += (size_t)S * slots * 4;
  if (kScore) b += (size_t)maxr * slots * 12;
  b += (size_t)block * 4 + 2 * (size_t)pool * (block / 32) * 4;
  return (b + 15) & ~(size_t)15;
}

__device__ inline SortedSmem carve(unsigned char* p, int blob_words, int S,
                                   int maxr, int pool, int block) {
  SortedSmem s;
  const int slots = pool * block;
  s.slots = slots;
  s.blob = (uint32_t*)p;
  p += (size_t)blob_words * 4;
  s.bar = (uint64_t*)p;
  p += 16;
  s.pk = (uint32_t*)p;
  p += packed_bytes(maxr);
  s.scratch = (int64_t*)p;
  p += (size_t)S * block * 8;
  s.t = (double*)p;
  p += slots * 8;
  s.n = (uint64_t*)p;
  p += slots * 8;
  s.events = (int64_t*)p;
  p += slots * 8;
  s.steps = (int64_t*)p;
  p += slots * 8;
  s.h = (uint64_t*)p;
  p += slots * 8;
  s.traj = (int64_t*)p;
  p += slots * 8;
  s.integ = (double*)p;
  if (kScore) p += (size_t)maxr * slots * 8;
  s.x = (int32_t*)p;
  p += (size_t)S * slots * 4;
  s.f = (int32_t*)p;
  p += slots * 4;
  s.leap_q = (uint32_t*)p;
  p += slots * 4;
  s.ssa_left = (int32_t*)p;
  p += slots * 4;
  s.flags = (int32_t*)p;
  p += slots * 4;
  s.cnt = (int32_t*)p;
  if (kScore) p += (size_t)maxr * slots * 4;
  s.run = (int32_t*)p;
  p += block * 4;
  s.gcnt = (int32_t*)p;
  return s;
}

__device__ __forceinline__ void load_state(const SortedSmem& s, int p,
                                           TState& st) {
  st.t = s.t[p];
  st.n = s.n[p];
  st.events = s.events[p];
  st.steps = s.steps[p];
  st.h = s.h[p];
  st.f = s.f[p];
  st.leap_q = s.leap_q[p];
  st.ssa_left = s.ssa_left[p];
  st.flags = s.flags[p];
}

__device__ __forceinline__ void store_state(const SortedSmem& s, int p,
                                            const TState& st) {
  s.t[p] = st.t;
  s.n[p] = st.n;
  s.events[p] = st.events;
  s.steps[p] = st.steps;
  s.h[p] = st.h;
  s.f[p] = st.f;
  s.leap_q[p] = st.leap_q;
  s.ssa_left[p] = st.ssa_left;
  s.flags[p] = st.flags;
}

// Put trajectory u (or nothing, u >= n_traj) into slot p.
template <int NACC>
__device__ __forceinline__ void fill_slot(const SortedSmem& s,
                                          const ModelView& m, int p,
                                          int64_t u, int64_t n_traj) {
  if (u < n_traj) {
    TState st;
    thread_init<true>(m, s.x + p, s.slots, st);
    store_state(s, p, st);
    s.traj[p] = u;
    if (kScore) {
#pragma unroll
      for (int j = 0; j < NACC; ++j) {
        s.integ[j * s.slots + p] = 0.0;
        s.cnt[j * s.slots + p] = 0;
      }
    }
  } else {
    s.traj[p] = -1;
  }
}

// NB: block size fixed at compile time, or 0 for blockDim.x.  PK:
// kPkPacked for models whose every reaction packs (the host checks), else
// kPkRuntime.  RX: MAXR when the model has exactly MAXR reactions (the
// host checks), else 0.
template <int MAXR, int NB, int PK, int RX = 0>
__global__ void __launch_bounds__(kMaxBlock, kMinBlocks)
    k_tau_sorted(const uint32_t* __restrict__ gblob, int blob_words,
                 int64_t n_traj, uint64_t id_base, RunArgs ra, OutBase ob,
                 unsigned long long* queue, int cap_ssa, int cap_leap,
                 int pool) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int S = (int)__ldg(gblob + PYST_H_S);
  const int nb = NB ? NB : blockDim.x, nw = nb >> 5;
  SortedSmem sm = carve(smem, blob_words, S, MAXR, pool, nb);
  const int slots = sm.slots, groups = pool * nw;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) {
    mbar_init(sm.bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const bool ok = stage_blob(sm.blob, gblob, blob_words, sm.bar, 0,
                             ra.stage_polls);
  // Initial fill: a balanced contiguous range per block when every
  // trajectory fits the pools, else full pools and the queue for the rest.
  const int64_t grid = gridDim.x;
  const bool full = n_traj >= grid * slots;
  const int64_t lo = full ? (int64_t)blockIdx.x * slots
                          : (int64_t)blockIdx.x * n_traj / grid;
  const int64_t hi = full ? lo + slots
                          : ((int64_t)blockIdx.x + 1) * n_traj / grid;
  const int64_t qbase = full ? grid * slots : n_traj;
  if (!ok) {
    mbar_drain(sm.bar, 0);
    for (int k = 0; k < pool; ++k) {
      const int64_t u = lo + k * nb + tid;
      if (u < hi) mark_staging_failure(ob, u);
    }
    int64_t u = qbase + (int64_t)atomicAdd(queue, 1ull);
    while (u < n_traj) {
      mark_staging_failure(ob, u);
      u = qbase + (int64_t)atomicAdd(queue, 1ull);
    }
    return;
  }
  ModelView m;
  m.load(sm.blob);
  const int R = m.R;
  if (MAXR > 0) {
    m.pk = sm.pk;
    m.fast = __syncthreads_and(pack_reactions(m, sm.pk)) != 0;
  }
  constexpr int kAcc = (kScore && MAXR > 0) ? MAXR : 1;
  for (int k = 0; k < pool; ++k) {
    const int p = k * nb + tid;
    const int64_t u = lo + p;
    fill_slot<kAcc>(sm, m, p, u < hi ? u : n_traj, n_traj);
  }
  const unsigned lt = (1u << lane) - 1u;
  int rot0 = 0, rot1 = 0;
  __syncthreads();

  while (true) {
    // ---- schedule: counting sort of the slots by (SSA, leap, empty) ----
    int key[kMaxPool];
    unsigned b0[kMaxPool], b1[kMaxPool];
#pragma unroll
    for (int k = 0; k < kMaxPool; ++k) {
      if (k >= pool) break;
      const int p = k * nb + tid;
      key[k] = sm.traj[p] < 0 ? 2 : ((sm.flags[p] & TS_LEAPGRP) ? 1 : 0);
      b0[k] = __ballot_sync(0xffffffffu, key[k] == 0);
      b1[k] = __ballot_sync(0xffffffffu, key[k] == 1);
      if (lane == 0) {
        sm.gcnt[k * nw + wid] = __popc(b0[k]);
        sm.gcnt[groups + k * nw + wid] = __popc(b1[k]);
      }
    }
    __syncthreads();
    int tot0 = 0, tot1 = 0, pre0[kMaxPool], pre1[kMaxPool];
    {
      // every warp scans the groups' counts itself: lane l holds groups l
      // and l + 32, the SSA count in the low and the leaping count in the
      // high 16 bits (a block's slots, at most 2048, fit either half)
      const int ga = lane, gb = lane + 32;
      const int ca = ga < groups ? sm.gcnt[ga] | sm.gcnt[groups + ga] << 16
                                 : 0;
      const int cb = gb < groups ? sm.gcnt[gb] | sm.gcnt[groups + gb] << 16
                                 : 0;
      int va = ca, vb = cb;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int ta = __shfl_up_sync(0xffffffffu, va, d);
        const int tb = __shfl_up_sync(0xffffffffu, vb, d);
        if (lane >= d) {
          va += ta;
          vb += tb;
        }
      }
      vb += __shfl_sync(0xffffffffu, va, 31);
      const int tot = __shfl_sync(0xffffffffu, vb, 31);
      tot0 = tot & 0xffff;
      tot1 = tot >> 16;
      const int xa = va - ca, xb = vb - cb;  // exclusive prefixes
#pragma unroll
      for (int k = 0; k < kMaxPool; ++k) {
        const int g = k * nw + wid;  // warp-uniform
        const int pa = __shfl_sync(0xffffffffu, xa, g & 31);
        const int pb = __shfl_sync(0xffffffffu, xb, g & 31);
        const int pre = g < 32 ? pa : pb;
        pre0[k] = pre & 0xffff;
        pre1[k] = pre >> 16;
      }
    }
    if (tot0 + tot1 == 0) break;  // uniform: every thread read the same
    // how many slots of each mode run: all if they fit, else a split in
    // proportion to the counts, in whole warps, with at least one warp's
    // worth of a mode that has any slots
    int n0 = tot0, n1 = tot1;
    if (tot0 + tot1 > nb) {
      n0 = (int)(((int64_t)tot0 * nb / (tot0 + tot1) + 16) / 32 * 32);
      const int min0 = tot0 < 32 ? tot0 : 32;
      const int min1 = tot1 < 32 ? tot1 : 32;
      if (n0 < min0) n0 = min0;
      if (n0 > nb - min1) n0 = nb - min1;
      if (n0 > tot0) n0 = tot0;
      n1 = nb - n0;
      if (n1 > tot1) {
        n1 = tot1;
        n0 = nb - n1;
      }
    }
    if (tot0) rot0 %= tot0;
    if (tot1) rot1 %= tot1;
#pragma unroll
    for (int k = 0; k < kMaxPool; ++k) {
      if (k >= pool) break;
      const int p = k * nb + tid;
      if (key[k] == 0) {
        int pos = pre0[k] + __popc(b0[k] & lt) - rot0;
        if (pos < 0) pos += tot0;
        if (pos < n0) sm.run[pos] = p;
      } else if (key[k] == 1) {
        int pos = pre1[k] + __popc(b1[k] & lt) - rot1;
        if (pos < 0) pos += tot1;
        if (pos < n1) sm.run[n0 + pos] = p;
      }
    }
    rot0 += n0;
    rot1 += n1;
    __syncthreads();
    // ---- run ----
    const int nrun = n0 + n1;
    if (tid < nrun) {
      const int p = sm.run[tid];
      // the warp holding both modes (n0 inside it) runs half-length rounds
      const bool mixed = PYST_MIXED_HALF && n0 > wid * 32 &&
                         n0 < wid * 32 + 32 && nrun > n0;
      const int my_cap_ssa = mixed ? (cap_ssa + 1) / 2 : cap_ssa;
      const int my_cap_leap = mixed ? (cap_leap + 1) / 2 : cap_leap;
      TState st;
      load_state(sm, p, st);
      double integ[kAcc];
      int cnt[kAcc];
#pragma unroll
      for (int j = 0; j < kAcc; ++j) {
        integ[j] = kScore ? sm.integ[j * slots + p] : 0.0;
        cnt[j] = kScore ? sm.cnt[j * slots + p] : 0;
      }
      const int64_t u = sm.traj[p];
      const TrajOut o = ob.at(0, u, 0, 0, ob.stride, R);
      // each round's code for the slot's group only (warps are uniform
      // but for the one mixed warp, which diverges across the two calls)
      if (st.flags & TS_LEAPGRP)
        any_round<MAXR, true, kScore, PK, kGroupLeap, RX>(
            m, sm.x + p, sm.scratch + tid, slots, nb, ra,
            id_base + (uint64_t)u, st, integ, cnt, o, my_cap_ssa,
            my_cap_leap, true);
      else
        any_round<MAXR, true, kScore, PK, kGroupSsa, RX>(
            m, sm.x + p, sm.scratch + tid, slots, nb, ra,
            id_base + (uint64_t)u, st, integ, cnt, o, my_cap_ssa,
            my_cap_leap, true);
      if (st.flags & TS_DONE) {
        thread_finish<(MAXR > 0 ? MAXR : 1), kScore>(m, sm.x + p, slots, st,
                                                     integ, cnt, o);
        fill_slot<kAcc>(sm, m, p, qbase + (int64_t)atomicAdd(queue, 1ull),
                        n_traj);
      } else {
        store_state(sm, p, st);
        if (kScore) {
#pragma unroll
          for (int j = 0; j < kAcc; ++j) {
            sm.integ[j * slots + p] = integ[j];
            sm.cnt[j * slots + p] = cnt[j];
          }
        }
      }
    }
    __syncthreads();
  }
}

template <int MR>
int launch_one(const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
               uint64_t id_base, const RunArgs& ra, const OutBase& ob,
               unsigned long long* queue, cudaStream_t st,
               const SortedGeometry& g) {
  const int maxr = MR > 0 ? MR : 1;
  // the largest block (whole warps) up to the preferred size whose pools
  // fit, first with the preferred slots per thread, then with one
  const int pref_block = g.block ? (g.block < kMaxBlock ? g.block : kMaxBlock)
                                 : kPrefBlock;
  const int pref_pool = g.pool ? (g.pool < kMaxPool ? g.pool : kMaxPool)
                               : kMaxPool;
  static const int kBlocks[] = {896, 768, 640, 512, 448, 384, 320, 256,
                                224, 192, 160, 128, 96, 64};
  int pool = 0, block = 0;
  for (int p = pref_pool; p >= 1 && !block; --p)
    for (int b : kBlocks)
      if (b <= pref_block &&
          sorted_smem_bytes(mi.words, mi.S, maxr, p, b) <= kMaxDynSmem) {
        pool = p;
        block = b;
        break;
      }
  if (!block) return PYST_EUNSUPPORTED;
  const size_t smem = sorted_smem_bytes(mi.words, mi.S, maxr, pool, block);
  // compile-time packed descriptors when every reaction packs (MAXR > 0)
  constexpr int kPk = MR > 0 ? kPkPacked : kPkRuntime;
  auto kf = mi.packable
                ? (block == kMaxBlock ? k_tau_sorted<MR, kMaxBlock, kPk>
                                      : k_tau_sorted<MR, 0, kPk>)
                : (block == kMaxBlock ? k_tau_sorted<MR, kMaxBlock, kPkRuntime>
                                      : k_tau_sorted<MR, 0, kPkRuntime>);
  // a packable model with exactly MR reactions in the full-size block: the
  // reaction count fixed at compile time (Schlogl, R = 4: 64.0 -> 57.8 ms)
  if (MR > 0 && mi.packable && block == kMaxBlock && mi.R == MR)
    kf = k_tau_sorted<MR, kMaxBlock, kPk, MR>;
  // and the reaction counts between (2, 3 and 5 to 7), without scores
  if constexpr (!kScore && (MR == 4 || MR == 8)) {
    if (mi.packable && block == kMaxBlock) {
      if (MR == 4 && mi.R == 2) kf = k_tau_sorted<2, kMaxBlock, kPkPacked, 2>;
      if (MR == 4 && mi.R == 3) kf = k_tau_sorted<3, kMaxBlock, kPkPacked, 3>;
      if (MR == 8 && mi.R == 5) kf = k_tau_sorted<5, kMaxBlock, kPkPacked, 5>;
      if (MR == 8 && mi.R == 6) kf = k_tau_sorted<6, kMaxBlock, kPkPacked, 6>;
      if (MR == 8 && mi.R == 7) kf = k_tau_sorted<7, kMaxBlock, kPkPacked, 7>;
    }
  }
  const int rc = set_smem(kf, smem);
  if (rc) return rc;
  if (cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st) !=
      cudaSuccess)
    return PYST_ECUDA;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf, block, smem);
  if (per_sm < 1) per_sm = 1;
  // every resident block slot of the GPU, each with at least two warps'
  // worth of trajectories
  int64_t grid = (n + 63) / 64;
  const int64_t cap = (int64_t)num_sms() * per_sm;
  if (grid > cap) grid = cap;
  kf<<<(unsigned)grid, block, smem, st>>>(d_blob, mi.words, n, id_base, ra,
                                          ob, queue, g.cap_ssa, g.cap_leap,
                                          pool);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

}  // namespace (flavour)
using namespace PYST_CAT(sorted_flavour_, PYST_SCORE, );

int PYST_CAT(launch_tau_sorted_, PYST_SCORE, )(
    int maxr, const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
    uint64_t id_base, const RunArgs& ra, const OutBase& ob,
    unsigned long long* queue, const SortedGeometry& g, cudaStream_t st) {
  if (n <= 0) return PYST_OK;
#if !PYST_SCORE
  if (maxr > PYST_THREAD_MAX_REACTIONS)
    return launch_one<0>(d_blob, mi, n, id_base, ra, ob, queue, st, g);
#else
  if (maxr > PYST_THREAD_MAX_REACTIONS) return PYST_EUNSUPPORTED;
#endif
  if (maxr <= 4) return launch_one<4>(d_blob, mi, n, id_base, ra, ob, queue, st, g);
  if (maxr <= 8) return launch_one<8>(d_blob, mi, n, id_base, ra, ob, queue, st, g);
  if (maxr <= 16)
    return launch_one<16>(d_blob, mi, n, id_base, ra, ob, queue, st, g);
  return launch_one<32>(d_blob, mi, n, id_base, ra, ob, queue, st, g);
}

}  // namespace pyst
