// Declarations shared by the kernel translation units and the C ABI.
//
// Each kernel family is compiled several times with -DPYST_TAU=0/1 and
// -DPYST_SCORE=0/1 (see py_stoch_b200/build.py) so the instantiations
// build in parallel; each object defines the launcher named by
// PYST_LAUNCHER_NAME for its flavour.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pyst_engine.cuh"
#include "pystoch_b200.h"

namespace pyst {

// Outputs of a whole launch; at() offsets them to one trajectory.
struct OutBase {
  int32_t* samples;
  int64_t stride;
  uint8_t* status;
  int64_t* events;
  uint64_t* seqhash;
  double* t_final;
  double* score;
  double* stats;
  double* jac;

  __device__ __forceinline__ TrajOut at(int64_t sample_off, int64_t u,
                                        int64_t traj_off, int64_t score_off,
                                        int64_t stride_, int R) const {
    TrajOut o;
    o.samples = samples + sample_off + u;
    o.stride = stride_;
    const int64_t v = traj_off + u;
    o.status = status ? status + v : nullptr;
    o.events = events ? events + v : nullptr;
    o.seqhash = seqhash ? seqhash + v : nullptr;
    o.t_final = t_final ? t_final + v : nullptr;
    o.score = score ? score + score_off + u * (int64_t)R : nullptr;
    return o;
  }
};

__device__ __forceinline__ void mark_staging_failure(const OutBase& ob,
                                                     int64_t v) {
  if (ob.status) ob.status[v] = (uint8_t)PYST_TRAJ_STAGING;
}

struct HostModelInfo {
  int S, R, words;
  int nlaw;       // reactions with a general kinetic law
  bool packable;  // every reaction fits the packed descriptors (no laws)
};

constexpr size_t kMaxDynSmem = 227 * 1024;

// Shared memory of the packed reaction descriptors (pack_reactions): 2R
// words, rounded up to 16 bytes.
__host__ __device__ inline size_t packed_bytes(int R) {
  return ((size_t)R * 8 + 15) & ~(size_t)15;
}

inline size_t host_warp_bytes(int S, int R, bool score) {
  size_t b = (size_t)S * 8 + (size_t)S * 4 + (size_t)R * 4 + (size_t)R * 4 +
             (((size_t)R + 3) & ~(size_t)3);
  b = (b + 15) & ~(size_t)15;
  if (score) b += (size_t)R * 16;
  return b;
}

template <class K>
inline int set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) {
    if (cudaFuncSetAttribute(kernel,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)bytes) != cudaSuccess)
      return PYST_ECUDA;
  }
  return PYST_OK;
}

int num_sms();

// plain, one trajectory per thread (maxr = R; picks MAXR in {4,8,16,32})
#define PYST_DECL_THREAD(T, SC)                                              \
  int launch_plain_thread_##T##SC(int maxr, const uint32_t* d_blob,          \
                                  const HostModelInfo& mi, int64_t n,        \
                                  uint64_t id_base, const RunArgs& ra,       \
                                  const OutBase& ob, int bs,                 \
                                  unsigned long long* queue, cudaStream_t st);
PYST_DECL_THREAD(0, 0)
PYST_DECL_THREAD(0, 1)
PYST_DECL_THREAD(1, 0)
PYST_DECL_THREAD(1, 1)
#undef PYST_DECL_THREAD

#define PYST_DECL_WARP(T, SC)                                                \
  int launch_plain_warp_##T##SC(const uint32_t* d_blob,                      \
                                const HostModelInfo& mi, int64_t n,          \
                                uint64_t id_base, const RunArgs& ra,         \
                                const OutBase& ob, int bs,                   \
                                unsigned long long* queue, cudaStream_t st);
PYST_DECL_WARP(0, 0)
PYST_DECL_WARP(0, 1)
PYST_DECL_WARP(1, 0)
PYST_DECL_WARP(1, 1)
#undef PYST_DECL_WARP

#define PYST_DECL_BATCH(SC)                                                  \
  int launch_batch_##SC(const uint32_t* d_blobs,                             \
                        const pyst_batch_item* d_items, int64_t n_items,     \
                        const pyst_batch_limits* lim, const RunArgs& ra,     \
                        const OutBase& ob, unsigned long long* queue,       \
                        unsigned* done, int bs, cudaStream_t st);
PYST_DECL_BATCH(0)
PYST_DECL_BATCH(1)
#undef PYST_DECL_BATCH

// Geometry of the mode-sorted kernel: round lengths, and the preferred
// slots per thread and block size (0: the kernel's defaults).
struct SortedGeometry {
  int cap_ssa, cap_leap, pool, block;
};

#define PYST_DECL_SORTED(SC)                                                 \
  int launch_tau_sorted_##SC(int maxr, const uint32_t* d_blob,               \
                             const HostModelInfo& mi, int64_t n,             \
                             uint64_t id_base, const RunArgs& ra,            \
                             const OutBase& ob, unsigned long long* queue,   \
                             const SortedGeometry& g, cudaStream_t st);
PYST_DECL_SORTED(0)
PYST_DECL_SORTED(1)
#undef PYST_DECL_SORTED

int launch_score_backward(const int32_t* samples, const double* score,
                          int64_t U, int kappa, int ita, int R,
                          const double* mean, const double* var,
                          const double* gmean, const double* gvar,
                          double* part, double* grad, cudaStream_t st);
int64_t score_backward_blocks(int64_t U);
int launch_score_partials(const int32_t* samples, const double* score,
                          int64_t U, int kappa, int ita, int R,
                          const double* mean, const double* var,
                          const double* gmean, const double* gvar,
                          double* part, cudaStream_t st);
int launch_score_combine(const double* part, int64_t nblk, int R,
                         int64_t n_total, double* grad, cudaStream_t st);
int launch_sample_sums(const int32_t* samples, int64_t U, int64_t stride,
                       int rows, int64_t* sums, cudaStream_t st);
int launch_moments_from_sums(const int64_t* sums, int rows, int64_t n,
                             double* mean, double* var, cudaStream_t st);

}  // namespace pyst

#define PYST_CAT2(a, b, c) a##b##c
#define PYST_CAT(a, b, c) PYST_CAT2(a, b, c)
