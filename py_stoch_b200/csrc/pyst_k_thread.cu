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

template <int MAXR, bool TAU, bool SCORE>
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
      run_thread<MAXR, TAU, SCORE>(m, xcol, slot, bs, ra,
                                   id_base + (uint64_t)u, o);
    u = nthreads + (int64_t)atomicAdd(queue, 1ull);
  }
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
// runs of at most this many trajectories per SM take the lane groups
constexpr int kGroupMaxPerSm = 16;

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

template <int MR>
int launch_one(const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
               uint64_t id_base, const RunArgs& ra, const OutBase& ob, int bs,
               cudaStream_t st, size_t smem, unsigned long long* queue) {
  auto kf = k_plain_thread<MR, (bool)PYST_TAU, (bool)PYST_SCORE>;
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
  // fewer trajectories than one 128-thread block of lane groups per SM
  if (maxr <= 8 && bs <= 128 && bs % kGroupLanes == 0 &&
      n <= (int64_t)num_sms() * kGroupMaxPerSm) {
    if (maxr <= 4)
      return launch_group<4>(d_blob, mi, n, id_base, ra, ob, bs, st, smem);
    return launch_group<8>(d_blob, mi, n, id_base, ra, ob, bs, st, smem);
  }
#endif
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
