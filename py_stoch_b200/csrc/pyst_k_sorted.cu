// Mode-sorted persistent kernel for thread-mapped tau-leaping.
//
// In tau-leaping each trajectory is, at any time, either in an SSA
// fallback round (mod/simulator/cuTauLeaping/P3.py:71-151) or leaping
// (P1_P2.py:96-297).  The reference runs the two as separate kernels, so in
// each launch the threads of the other mode sit idle.  Here a block keeps
// its trajectories' state in shared-memory slots and runs in rounds: every
// thread advances the trajectory in its slot for up to cap_ssa SSA steps or
// cap_leap leaps (stopping early when a DECIDE switches mode); between
// rounds the block refills finished slots from the global work queue and
// counting-sorts the slots by mode, so each warp executes one kind of step.
// Per-trajectory arithmetic is exactly that of run_thread, so results do not
// depend on the schedule.  Built once per PYST_SCORE flavour.
#include "pyst_launch.cuh"

namespace pyst {
// see pyst_k_thread.cu: per-flavour namespace, not an anonymous one
namespace PYST_CAT(sorted_flavour_, PYST_SCORE, ) {

constexpr bool kScore = (bool)PYST_SCORE;
constexpr int kBlock = kScore ? 128 : 256;

// Blocks per SM the register allocation must allow (launch bounds); 4
// (at most 64 registers) measured fastest on B200 for the Schlogl
// workload, ahead of 3 (85) and 1 (unbounded, 111).
#ifndef PYST_SORTED_MINB
#define PYST_SORTED_MINB 4
#endif
// Round length in SM clock cycles (0: rounds end only on the step caps).
// A time box makes the warps of a block reach the regrouping barrier
// together whatever mix of SSA steps and leaps they run.
#ifndef PYST_ROUND_CYCLES
#define PYST_ROUND_CYCLES 0
#endif
// Cooperative round end: a thread at its step cap keeps stepping until
// every active thread of the block has reached its cap or stopped, so
// warps do not idle at the regrouping barrier.  Off: on the Schlogl
// workload it measured 1.48x slower (316 vs 214 ms) -- the warps that keep
// stepping take issue slots from the slowest warp and stretch the round.
#ifndef PYST_MIXED_HALF
#define PYST_MIXED_HALF 1
#endif
#ifndef PYST_COOP_ROUNDS
#define PYST_COOP_ROUNDS 0
#endif

struct SortedSmem {
  uint32_t* blob;
  uint64_t* bar;
  int32_t* xa;
  int32_t* xb;
  int64_t* slot;
  double* t;
  uint64_t* n;
  int64_t* events;
  int64_t* steps;
  uint64_t* h;
  int64_t* traj;
  int32_t* f;
  uint32_t* leap_q;
  int32_t* ssa_left;
  int32_t* flags;
  double* integ;  // [MAXR][kBlock]
  int32_t* cnt;   // [MAXR][kBlock]
  int32_t* wcnt;  // [2][warps]
};

__host__ __device__ inline size_t sorted_smem_bytes(int blob_words, int S,
                                                    int maxr) {
  size_t b = (size_t)blob_words * 4 + 16;
  b += (size_t)S * kBlock * 4 * 2;  // xa, xb
  b += (size_t)S * kBlock * 8;      // slot
  b += (size_t)kBlock * (8 * 6 + 4 * 4);
  if (kScore) b += (size_t)maxr * kBlock * 12;
  b += 2 * (kBlock / 32) * 4;
  return (b + 15) & ~(size_t)15;
}

__device__ inline SortedSmem carve(unsigned char* p, int blob_words, int S,
                                   int maxr) {
  SortedSmem s;
  s.blob = (uint32_t*)p;
  p += (size_t)blob_words * 4;
  s.bar = (uint64_t*)p;
  p += 16;
  s.slot = (int64_t*)p;
  p += (size_t)S * kBlock * 8;
  s.t = (double*)p;
  p += kBlock * 8;
  s.n = (uint64_t*)p;
  p += kBlock * 8;
  s.events = (int64_t*)p;
  p += kBlock * 8;
  s.steps = (int64_t*)p;
  p += kBlock * 8;
  s.h = (uint64_t*)p;
  p += kBlock * 8;
  s.traj = (int64_t*)p;
  p += kBlock * 8;
  s.integ = (double*)p;
  if (kScore) p += (size_t)maxr * kBlock * 8;
  s.xa = (int32_t*)p;
  p += (size_t)S * kBlock * 4;
  s.xb = (int32_t*)p;
  p += (size_t)S * kBlock * 4;
  s.f = (int32_t*)p;
  p += kBlock * 4;
  s.leap_q = (uint32_t*)p;
  p += kBlock * 4;
  s.ssa_left = (int32_t*)p;
  p += kBlock * 4;
  s.flags = (int32_t*)p;
  p += kBlock * 4;
  s.cnt = (int32_t*)p;
  if (kScore) p += (size_t)maxr * kBlock * 4;
  s.wcnt = (int32_t*)p;
  return s;
}

template <int MAXR>
__global__ void __launch_bounds__(kBlock, PYST_SORTED_MINB)
    k_tau_sorted(const uint32_t* __restrict__ gblob, int blob_words,
                 int64_t n_traj, uint64_t id_base, RunArgs ra, OutBase ob,
                 unsigned long long* queue, int cap_ssa, int cap_leap) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int S = (int)__ldg(gblob + PYST_H_S);
  SortedSmem sm = carve(smem, blob_words, S, MAXR);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int nw = kBlock / 32;
  if (tid == 0) {
    mbar_init(sm.bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const bool ok = stage_blob(sm.blob, gblob, blob_words, sm.bar, 0);
  const int64_t nthreads = (int64_t)gridDim.x * kBlock;
  int64_t u = blockIdx.x * (int64_t)kBlock + tid;
  if (!ok) {
    mbar_wait(sm.bar, 0);
    while (u < n_traj) {
      mark_staging_failure(ob, u);
      u = nthreads + (int64_t)atomicAdd(queue, 1ull);
    }
    return;
  }
  ModelView m;
  m.load(sm.blob);
  const int R = m.R;
  int32_t* xa = sm.xa;
  int32_t* xb = sm.xb;
  int64_t* slotc = sm.slot + tid;
  TState st;
  constexpr int kAcc = (kScore && MAXR > 0) ? MAXR : 1;
  double integ[kAcc];
  int cnt[kAcc];
  auto zero_score = [&]() {
#pragma unroll
    for (int j = 0; j < kAcc; ++j) {
      integ[j] = 0.0;
      cnt[j] = 0;
    }
  };
  bool active = u < n_traj;
  zero_score();
  if (active) thread_init<true>(m, xa + tid, kBlock, st);
  else st.flags = TS_DONE;
  const unsigned lt = (1u << lane) - 1u;
  __shared__ int s_reached;
  if (tid == 0) s_reached = 0;
  int n_active = __syncthreads_count(active);

  // After sorting, at most one warp per block holds both SSA and leaping
  // slots and executes both code paths in turn; it runs rounds of half
  // length so it reaches the regrouping barrier with the pure warps.
  int my_cap_ssa = cap_ssa, my_cap_leap = cap_leap;
  while (true) {
    if (active) {
      const TrajOut o = ob.at(0, u, 0, 0, ob.stride, R);
      const long long deadline =
          PYST_ROUND_CYCLES ? (long long)clock64() + PYST_ROUND_CYCLES : 0;
      any_round<MAXR, true, kScore>(m, xa + tid, slotc, kBlock, ra,
                                    id_base + (uint64_t)u, st, integ, cnt, o,
                                    my_cap_ssa, my_cap_leap, true, deadline,
                                    PYST_COOP_ROUNDS ? &s_reached : nullptr,
                                    n_active);
      if (st.flags & TS_DONE) {
        thread_finish<(MAXR > 0 ? MAXR : 1), kScore>(m, xa + tid, kBlock, st,
                                                     integ, cnt, o);
        u = nthreads + (int64_t)atomicAdd(queue, 1ull);
        active = u < n_traj;
        zero_score();
        if (active) thread_init<true>(m, xa + tid, kBlock, st);
      }
    }
    // ---- regroup: counting sort of the slots by (SSA, leap, empty) ----
    const int key = !active ? 2 : ((st.flags & TS_LEAPGRP) ? 1 : 0);
    const unsigned b0 = __ballot_sync(0xffffffffu, key == 0);
    const unsigned b1 = __ballot_sync(0xffffffffu, key == 1);
    if (lane == 0) {
      sm.wcnt[wid] = __popc(b0);
      sm.wcnt[nw + wid] = __popc(b1);
    }
    __syncthreads();
    int tot0 = 0, tot1 = 0, pre0 = 0, pre1 = 0, pre2 = 0;
#pragma unroll
    for (int w = 0; w < nw; ++w) {
      const int c0 = sm.wcnt[w], c1 = sm.wcnt[nw + w];
      tot0 += c0;
      tot1 += c1;
      if (w < wid) {
        pre0 += c0;
        pre1 += c1;
        pre2 += 32 - c0 - c1;
      }
    }
    if (tot0 + tot1 == 0) break;  // uniform: every thread read the same
    n_active = tot0 + tot1;
    if (tid == 0) s_reached = 0;  // read only after the next barrier
    int rank;
    if (key == 0) rank = pre0 + __popc(b0 & lt);
    else if (key == 1) rank = tot0 + pre1 + __popc(b1 & lt);
    else rank = tot0 + tot1 + pre2 + __popc(~(b0 | b1) & lt);
    // move this slot's state to position `rank`
    sm.t[rank] = st.t;
    sm.n[rank] = st.n;
    sm.events[rank] = st.events;
    sm.steps[rank] = st.steps;
    sm.h[rank] = st.h;
    sm.traj[rank] = active ? u : -1;
    sm.f[rank] = st.f;
    sm.leap_q[rank] = st.leap_q;
    sm.ssa_left[rank] = st.ssa_left;
    sm.flags[rank] = st.flags;
    for (int i = 0; i < S; ++i)
      xb[(int64_t)i * kBlock + rank] = xa[(int64_t)i * kBlock + tid];
    if (kScore) {
#pragma unroll
      for (int j = 0; j < kAcc; ++j) {
        sm.integ[j * kBlock + rank] = integ[j];
        sm.cnt[j * kBlock + rank] = cnt[j];
      }
    }
    __syncthreads();
    st.t = sm.t[tid];
    st.n = sm.n[tid];
    st.events = sm.events[tid];
    st.steps = sm.steps[tid];
    st.h = sm.h[tid];
    u = sm.traj[tid];
    st.f = sm.f[tid];
    st.leap_q = sm.leap_q[tid];
    st.ssa_left = sm.ssa_left[tid];
    st.flags = sm.flags[tid];
    if (kScore) {
#pragma unroll
      for (int j = 0; j < kAcc; ++j) {
        integ[j] = sm.integ[j * kBlock + tid];
        cnt[j] = sm.cnt[j * kBlock + tid];
      }
    }
    active = u >= 0;
    {
      const bool in_leap = active && (st.flags & TS_LEAPGRP);
      const bool in_ssa = active && !(st.flags & TS_LEAPGRP);
      const bool mixed = PYST_MIXED_HALF &&
                         __any_sync(0xffffffffu, in_leap) &&
                         __any_sync(0xffffffffu, in_ssa);
      my_cap_ssa = mixed ? (cap_ssa + 1) / 2 : cap_ssa;
      my_cap_leap = mixed ? (cap_leap + 1) / 2 : cap_leap;
    }
    int32_t* tmp = xa;
    xa = xb;
    xb = tmp;
  }
}

template <int MR>
int launch_one(const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
               uint64_t id_base, const RunArgs& ra, const OutBase& ob,
               unsigned long long* queue, cudaStream_t st, int cap_ssa,
               int cap_leap) {
  const size_t smem = sorted_smem_bytes(mi.words, mi.S, MR > 0 ? MR : 1);
  if (smem > kMaxDynSmem) return PYST_EUNSUPPORTED;
  auto kf = k_tau_sorted<MR>;
  const int rc = set_smem(kf, smem);
  if (rc) return rc;
  if (cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st) !=
      cudaSuccess)
    return PYST_ECUDA;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf, kBlock, smem);
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (n + kBlock - 1) / kBlock;
  const int64_t cap = (int64_t)num_sms() * per_sm;
  if (grid > cap) grid = cap;
  kf<<<(unsigned)grid, kBlock, smem, st>>>(d_blob, mi.words, n, id_base, ra,
                                           ob, queue, cap_ssa, cap_leap);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

}  // namespace (flavour)
using namespace PYST_CAT(sorted_flavour_, PYST_SCORE, );

int PYST_CAT(launch_tau_sorted_, PYST_SCORE, )(
    int maxr, const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
    uint64_t id_base, const RunArgs& ra, const OutBase& ob,
    unsigned long long* queue, int cap_ssa, int cap_leap, cudaStream_t st) {
  if (n <= 0) return PYST_OK;
#if !PYST_SCORE
  if (maxr > PYST_THREAD_MAX_REACTIONS)
    return launch_one<0>(d_blob, mi, n, id_base, ra, ob, queue, st, cap_ssa,
                         cap_leap);
#else
  if (maxr > PYST_THREAD_MAX_REACTIONS) return PYST_EUNSUPPORTED;
#endif
  if (maxr <= 4)
    return launch_one<4>(d_blob, mi, n, id_base, ra, ob, queue, st, cap_ssa,
                         cap_leap);
  if (maxr <= 8)
    return launch_one<8>(d_blob, mi, n, id_base, ra, ob, queue, st, cap_ssa,
                         cap_leap);
  if (maxr <= 16)
    return launch_one<16>(d_blob, mi, n, id_base, ra, ob, queue, st, cap_ssa,
                          cap_leap);
  return launch_one<32>(d_blob, mi, n, id_base, ra, ob, queue, st, cap_ssa,
                        cap_leap);
}

}  // namespace pyst
