// Likelihood-ratio gradient reduction and the test hooks.
#include <curand_kernel.h>

#include <mutex>

#include "pyst_launch.cuh"
#include "pystoch_b200_testing.h"

namespace pyst {
namespace {

#define PYST_BWD_CHUNK 256

// h_u for a chunk of trajectories, then per-block partial sums
// part[block][j] = sum_{u in chunk} h_u score[u][j] in trajectory order.
__global__ void __launch_bounds__(PYST_BWD_CHUNK)
    k_score_partial(const int32_t* __restrict__ samples,
                    const double* __restrict__ score, int64_t U, int kappa,
                    int ita, int R, const double* __restrict__ mean,
                    const double* __restrict__ var,
                    const double* __restrict__ gmean,
                    const double* __restrict__ gvar, double* part) {
  __shared__ double hs[PYST_BWD_CHUNK];
  const int64_t u0 = blockIdx.x * (int64_t)PYST_BWD_CHUNK;
  const int64_t u = u0 + threadIdx.x;
  double h = 0.0;
  if (u < U) {
    const int KF = kappa * ita;
    for (int kf = 0; kf < KF; ++kf) {
      const double d =
          __dsub_rn((double)samples[(int64_t)kf * U + u], mean[kf]);
      h = __dadd_rn(h, __dmul_rn(gmean[kf], d));
      if (gvar)
        h = __dadd_rn(
            h, __dmul_rn(gvar[kf], __dsub_rn(__dmul_rn(d, d), var[kf])));
    }
  }
  hs[threadIdx.x] = h;
  __syncthreads();
  const int64_t rem = U - u0;
  const int n = (int)(rem < PYST_BWD_CHUNK ? rem : PYST_BWD_CHUNK);
  for (int j = threadIdx.x; j < R; j += PYST_BWD_CHUNK) {
    double acc = 0.0;
    for (int q = 0; q < n; ++q)
      acc = __dadd_rn(acc, __dmul_rn(hs[q], score[(u0 + q) * R + j]));
    part[(int64_t)blockIdx.x * R + j] = acc;
  }
}

__global__ void k_score_final(const double* __restrict__ part, int64_t nblk,
                              int R, int64_t U, double* grad) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < R;
       j += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int64_t b = 0; b < nblk; ++b)
      acc = __dadd_rn(acc, part[b * R + j]);
    grad[j] = __ddiv_rn(acc, (double)U);
  }
}

// Exact integer sufficient statistics of sample rows: for row kf (of
// kappa*ita) and the trajectories of this block's chunk, sum x, and x^2
// split into its high and low 32-bit halves (x^2 < 2^62), all added with
// 64-bit integer atomics into the zeroed sums[kf][3].  Integer sums are
// exact, so the result does not depend on the order of the additions, on
// the chunking or on how trajectories are split across GPUs.
#define PYST_SUMS_CHUNK 4096
__global__ void __launch_bounds__(256)
    k_sample_sums(const int32_t* __restrict__ samples, int64_t U,
                  int64_t stride, int rows, unsigned long long* sums) {
  __shared__ unsigned long long red[3][256];
  const int64_t u0 = (int64_t)blockIdx.x * PYST_SUMS_CHUNK;
  const int64_t u1 = u0 + PYST_SUMS_CHUNK < U ? u0 + PYST_SUMS_CHUNK : U;
  for (int kf = blockIdx.y; kf < rows; kf += gridDim.y) {
    const int32_t* row = samples + (int64_t)kf * stride;
    unsigned long long sx = 0, hi = 0, lo = 0;
    for (int64_t u = u0 + threadIdx.x; u < u1; u += 256) {
      const int64_t x = row[u];
      const unsigned long long x2 = (unsigned long long)(x * x);
      sx += (unsigned long long)x;  // two's complement: signed sum mod 2^64
      hi += x2 >> 32;
      lo += x2 & 0xFFFFFFFFull;
    }
    red[0][threadIdx.x] = sx;
    red[1][threadIdx.x] = hi;
    red[2][threadIdx.x] = lo;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
      if (threadIdx.x < w) {
        red[0][threadIdx.x] += red[0][threadIdx.x + w];
        red[1][threadIdx.x] += red[1][threadIdx.x + w];
        red[2][threadIdx.x] += red[2][threadIdx.x + w];
      }
      __syncthreads();
    }
    if (threadIdx.x < 3)
      atomicAdd(sums + 3 * (int64_t)kf + threadIdx.x, red[threadIdx.x][0]);
    __syncthreads();  // red is rewritten for the next row
  }
}

// Population mean and variance of each row from its exact sums over n
// trajectories: mean = sx / n, var = (hi 2^32 + lo) / n - mean^2.
__global__ void k_moments_from_sums(const long long* __restrict__ sums,
                                    int rows, int64_t n, double* mean,
                                    double* var) {
  const int kf = blockIdx.x * blockDim.x + threadIdx.x;
  if (kf >= rows) return;
  const double dn = (double)n;
  const double m = __ddiv_rn((double)sums[3 * kf], dn);
  const double x2 = __dadd_rn(__dmul_rn((double)sums[3 * kf + 1],
                                        4294967296.0),
                              (double)sums[3 * kf + 2]);
  mean[kf] = m;
  var[kf] = __dsub_rn(__ddiv_rn(x2, dn), __dmul_rn(m, m));
}

__global__ void k_philox(uint64_t seed, uint64_t id, uint64_t n0,
                         int64_t count, uint32_t* out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  Stream s = make_stream(seed, id);
  s.n = n0 + (uint64_t)i;
  const uint4 r = next_block(s);
  out[4 * i + 0] = r.x;
  out[4 * i + 1] = r.y;
  out[4 * i + 2] = r.z;
  out[4 * i + 3] = r.w;
}

__global__ void k_philox_raw(const uint32_t* ctr_key, int64_t count,
                             uint32_t* out, int use_curand) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t* c = ctr_key + 6 * i;
  uint4 r;
  if (use_curand)
    r = curand_Philox4x32_10(make_uint4(c[0], c[1], c[2], c[3]),
                             make_uint2(c[4], c[5]));
  else
    r = philox4x32_10(c[0], c[1], c[2], c[3], c[4], c[5]);
  out[4 * i + 0] = r.x;
  out[4 * i + 1] = r.y;
  out[4 * i + 2] = r.z;
  out[4 * i + 3] = r.w;
}

__global__ void k_math(const double* x, int64_t n, int which, double* out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = 0.0;
  if (which == 0) v = pyst_log(x[i]);
  else if (which == 1) v = pyst_exp(x[i]);
  else if (which == 2) v = pyst_logfact(x[i]);
  else if (which == 3) v = log(x[i]);
  else if (which == 4) v = exp(x[i]);
  out[i] = v;
}

__global__ void k_poisson(const float* lam, int64_t n, uint64_t seed,
                          int32_t* out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Stream s = make_stream(seed, (uint64_t)i);
  out[i] = poisson(lam[i], leap_key(s, 7u, (int)(i & 1023), 3));
}

// Issue-rate probe of one arithmetic pipe: 8 independent dependency chains
// per thread, so the pipe, not latency, bounds it.  OP 0: FP32 fused
// multiply-add; 1: INT32 multiply-add (mad.lo.u32); 2: FP64 fused
// multiply-add; 3: INT32 xor-shift-add (the ALU forms Philox's xors and
// key additions use).  One operation per chain per iteration.
template <int OP>
__global__ void __launch_bounds__(256) k_pipe(int iters, double* sink) {
  const uint32_t t = blockIdx.x * 256u + threadIdx.x;
  float f[8];
  uint32_t x[8];
  double d[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    f[c] = (float)(t + c) * 1e-3f;
    x[c] = t * 8u + (uint32_t)c;
    d[c] = (double)(t + c) * 1e-3;
  }
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      if (OP == 0) f[c] = __fmaf_rn(f[c], 0.99999f, 1e-7f);
      // (integer chains in inline PTX: the compiler may not fold two
      // steps of a multiply-add chain into one)
      if (OP == 1)
        asm volatile("mad.lo.u32 %0, %0, %1, %2;"
                     : "+r"(x[c])
                     : "r"(0x9E3779B1u), "r"(0x7F4A7C15u));
      if (OP == 2) d[c] = __fma_rn(d[c], 0.99999, 1e-9);
      if (OP == 3)
        asm volatile("xor.b32 %0, %0, %1;\n\tadd.u32 %0, %0, %2;"
                     : "+r"(x[c])
                     : "r"((uint32_t)i), "r"(0x7F4A7C15u));
    }
  }
  double acc = 0.0;
#pragma unroll
  for (int c = 0; c < 8; ++c)
    acc = __dadd_rn(acc, OP == 0 ? (double)f[c]
                         : OP == 2 ? d[c] : (double)x[c]);
  sink[t] = acc;
}

}  // namespace

int64_t score_backward_blocks(int64_t U) {
  return (U + PYST_BWD_CHUNK - 1) / PYST_BWD_CHUNK;
}

int launch_score_backward(const int32_t* samples, const double* score,
                          int64_t U, int kappa, int ita, int R,
                          const double* mean, const double* var,
                          const double* gmean, const double* gvar,
                          double* part, double* grad, cudaStream_t st) {
  const int64_t nblk = score_backward_blocks(U);
  k_score_partial<<<(unsigned)nblk, PYST_BWD_CHUNK, 0, st>>>(
      samples, score, U, kappa, ita, R, mean, var, gmean, gvar, part);
  k_score_final<<<(R + 127) / 128, 128, 0, st>>>(part, nblk, R, U, grad);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

int launch_score_partials(const int32_t* samples, const double* score,
                          int64_t U, int kappa, int ita, int R,
                          const double* mean, const double* var,
                          const double* gmean, const double* gvar,
                          double* part, cudaStream_t st) {
  const int64_t nblk = score_backward_blocks(U);
  k_score_partial<<<(unsigned)nblk, PYST_BWD_CHUNK, 0, st>>>(
      samples, score, U, kappa, ita, R, mean, var, gmean, gvar, part);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

int launch_score_combine(const double* part, int64_t nblk, int R,
                         int64_t n_total, double* grad, cudaStream_t st) {
  k_score_final<<<(R + 127) / 128, 128, 0, st>>>(part, nblk, R, n_total,
                                                 grad);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

int launch_sample_sums(const int32_t* samples, int64_t U, int64_t stride,
                       int rows, int64_t* sums, cudaStream_t st) {
  if (cudaMemsetAsync(sums, 0, (size_t)rows * 3 * sizeof(int64_t), st) !=
      cudaSuccess)
    return PYST_ECUDA;
  if (U == 0) return PYST_OK;
  const dim3 grid((unsigned)((U + PYST_SUMS_CHUNK - 1) / PYST_SUMS_CHUNK),
                  (unsigned)(rows < 65535 ? rows : 65535));
  k_sample_sums<<<grid, 256, 0, st>>>(samples, U, stride, rows,
                                      (unsigned long long*)sums);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

int launch_moments_from_sums(const int64_t* sums, int rows, int64_t n,
                             double* mean, double* var, cudaStream_t st) {
  k_moments_from_sums<<<(rows + 127) / 128, 128, 0, st>>>(
      (const long long*)sums, rows, n, mean, var);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

// ---- allocation-free gradient reduction --------------------------------
// Scratch of pyst_score_backward_noalloc: the per-block partial sums live in
// this fixed array instead of caller workspace.  Every GPU that loads the
// library holds PYST_NOALLOC_SCRATCH_BYTES of it until the process exits.
static __device__ __align__(256) double
    g_noalloc_scratch[PYST_NOALLOC_SCRATCH_BYTES / sizeof(double)];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device.  On the host
// the symbol is only a stand-in; a kernel must be given this address.
// Looked up once per device, the first time the entry point runs there.
int noalloc_scratch(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return PYST_ECUDA;
  if (dev < 0 || dev >= kMaxDevices) return PYST_EUNSUPPORTED;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
      return PYST_ECUDA;
    g_noalloc_ptr[dev] = (double*)p;
  }
  *out = g_noalloc_ptr[dev];
  return PYST_OK;
}

}  // namespace

}  // namespace pyst

using namespace pyst;

extern "C" {

int pyst_score_backward_noalloc(const int32_t* samples, const double* score,
                                int64_t n_traj, int32_t kappa, int32_t ita,
                                int32_t n_reactions, const double* mean,
                                const double* var, const double* gmean,
                                const double* gvar, double* d_grad,
                                void* stream) {
  if (!samples || !score || !mean || !gmean || !d_grad || n_traj < 1 ||
      kappa < 1 || ita < 1 || n_reactions < 1)
    return PYST_EINVAL;
  if (gvar && !var) return PYST_EINVAL;
  const int64_t nblk = score_backward_blocks(n_traj);
  if ((uint64_t)nblk * (uint64_t)n_reactions * sizeof(double) >
      (uint64_t)PYST_NOALLOC_SCRATCH_BYTES)
    return PYST_EUNSUPPORTED;
  double* part = nullptr;
  const int rc = noalloc_scratch(&part);
  if (rc) return rc;
  return launch_score_backward(samples, score, n_traj, kappa, ita,
                               n_reactions, mean, var, gmean, gvar, part,
                               d_grad, (cudaStream_t)stream);
}

int pyst_test_pipe(int32_t which, int32_t iters, int32_t blocks,
                   double* d_sink, void* stream) {
  if (!d_sink || iters < 1 || blocks < 1 || which < 0 || which > 3)
    return PYST_EINVAL;
  cudaStream_t st = (cudaStream_t)stream;
  if (which == 0) k_pipe<0><<<blocks, 256, 0, st>>>(iters, d_sink);
  if (which == 1) k_pipe<1><<<blocks, 256, 0, st>>>(iters, d_sink);
  if (which == 2) k_pipe<2><<<blocks, 256, 0, st>>>(iters, d_sink);
  if (which == 3) k_pipe<3><<<blocks, 256, 0, st>>>(iters, d_sink);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

int pyst_test_philox(uint64_t seed, uint64_t id, uint64_t n0, int64_t count,
                     uint32_t* d_out, void* stream) {
  if (count <= 0) return PYST_OK;
  if (!d_out) return PYST_EINVAL;
  k_philox<<<(unsigned)((count + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
      seed, id, n0, count, d_out);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

int pyst_test_philox_raw(const uint32_t* d_ctr_key, int64_t count,
                         uint32_t* d_out, int use_curand, void* stream) {
  if (count <= 0) return PYST_OK;
  if (!d_ctr_key || !d_out) return PYST_EINVAL;
  k_philox_raw<<<(unsigned)((count + 127) / 128), 128, 0,
                 (cudaStream_t)stream>>>(d_ctr_key, count, d_out, use_curand);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

int pyst_test_math(const double* d_x, int64_t n, int which, double* d_out,
                   void* stream) {
  if (n <= 0) return PYST_OK;
  if (!d_x || !d_out || which < 0 || which > 4) return PYST_EINVAL;
  k_math<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
      d_x, n, which, d_out);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

int pyst_test_poisson(const float* d_lam, int64_t n, uint64_t seed,
                      int32_t* d_out, void* stream) {
  if (n <= 0) return PYST_OK;
  if (!d_lam || !d_out) return PYST_EINVAL;
  k_poisson<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(
      d_lam, n, seed, d_out);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

}  // extern "C"
