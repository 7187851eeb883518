// One-trajectory-per-warp kernel for a single model (large reaction
// counts).  Grid-stride over trajectories; built once per (PYST_TAU,
// PYST_SCORE) flavour.
#include "pyst_launch.cuh"

namespace pyst {
// nvcc gives template functions of an anonymous namespace weak external
// linkage on the host side, so the flavours built from this file would be
// merged at link time; a per-flavour namespace keeps them apart.
namespace PYST_CAT(warp_flavour_, PYST_TAU, PYST_SCORE) {

template <bool TAU, bool SCORE>
__global__ void __launch_bounds__(128)
    k_plain_warp(const uint32_t* __restrict__ gblob, int blob_words,
                 int64_t n_traj, uint64_t id_base, RunArgs ra, OutBase ob,
                 int warp_bytes, unsigned long long* queue) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* sblob = (uint32_t*)smem;
  uint64_t* bar = (uint64_t*)(smem + (size_t)blob_words * 4);
  unsigned char* wbase = smem + (size_t)blob_words * 4 + 16;
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const int nw = blockDim.x >> 5, wid = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * nw;
  const bool ok = stage_blob(sblob, gblob, blob_words, bar, 0,
                             ra.stage_polls);
  int64_t u = blockIdx.x * (int64_t)nw + wid;
  auto next = [&]() {
    long long v = 0;
    if (lane == 0) v = (long long)atomicAdd(queue, 1ull);
    return nwarps + (int64_t)__shfl_sync(0xffffffffu, v, 0);
  };
  if (!ok) {
    mbar_drain(bar, 0);
    while (u < n_traj) {
      if (lane == 0) mark_staging_failure(ob, u);
      u = next();
    }
    return;
  }
  ModelView m;
  m.load(sblob);
  unsigned char* mine = wbase + (size_t)wid * warp_bytes;
  const WarpSmem ws = warp_smem(mine, m.S, m.R);
  double* sacc = (double*)(mine + warp_smem_bytes(m.S, m.R));
  while (u < n_traj) {
    const TrajOut o = ob.at(0, u, 0, 0, ob.stride, m.R);
    run_warp<TAU, SCORE>(m, ws, ra, id_base + (uint64_t)u, o, sacc);
    u = next();
  }
}

}  // namespace (flavour)
using namespace PYST_CAT(warp_flavour_, PYST_TAU, PYST_SCORE);

int PYST_CAT(launch_plain_warp_, PYST_TAU, PYST_SCORE)(
    const uint32_t* d_blob, const HostModelInfo& mi, int64_t n,
    uint64_t id_base, const RunArgs& ra, const OutBase& ob, int bs,
    unsigned long long* queue, cudaStream_t st) {
  const int nw = bs / 32;
  const size_t wb = host_warp_bytes(mi.S, mi.R, PYST_SCORE);
  const size_t smem = (size_t)mi.words * 4 + 16 + wb * nw;
  if (smem > kMaxDynSmem) return PYST_EUNSUPPORTED;
  if (n <= 0) return PYST_OK;
  auto kf = k_plain_warp<(bool)PYST_TAU, (bool)PYST_SCORE>;
  const int rc = set_smem(kf, smem);
  if (rc) return rc;
  if (cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st) !=
      cudaSuccess)
    return PYST_ECUDA;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf, bs, smem);
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (n + nw - 1) / nw;
  const int64_t cap = (int64_t)num_sms() * per_sm;
  if (grid > cap) grid = cap;
  kf<<<(unsigned)grid, bs, smem, st>>>(d_blob, mi.words, n, id_base, ra, ob,
                                       (int)wb, queue);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

}  // namespace pyst
