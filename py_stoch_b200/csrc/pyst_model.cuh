// Device view of a packed model blob and its staging into shared memory.
//
// The blob (layout: include/pystoch_b200.h, PYST_H_*) replaces the
// reference's per-model __constant__ symbols d_A, d_V, d_H, d_H_type, d_c,
// d_I, d_E, d_x_0 (mod/simulator/cuTauLeaping/cuTauLeaping.py:86-107,
// mod/simulator/cuGillespie/cuGillespie.py:49-63) and the macros baked in by
// string.Template (cuTauLeaping.py:142-160).  One generic kernel serves
// every model: the blob is copied into shared memory with one bulk-async
// (TMA) copy per block, completion tracked by an mbarrier.
#pragma once
#include <stdint.h>

#include "pystoch_b200.h"

namespace pyst {

struct ModelView {
  const uint32_t* w;
  int S, R, kappa, ita;
  int o_rate, o_facptr, o_fac, o_netptr, o_net, o_times, o_out, o_x0;
  int o_spvptr, o_spv, o_g, o_critptr, o_crit;
  int o_lawptr, o_law, o_lawc, nlaw;  // general kinetic laws (nlaw = 0: none)
  int n_c;
  float eta;
  double t_max;
  // Packed per-reaction descriptors (see pack_reactions), valid when
  // `fast`: factors of reaction j at pk[j], net changes at pk[R + j].
  const uint32_t* pk;
  bool fast;

  __device__ __forceinline__ void load(const uint32_t* base) {
    w = base;
    S = (int)w[PYST_H_S];
    R = (int)w[PYST_H_R];
    kappa = (int)w[PYST_H_KAPPA];
    ita = (int)w[PYST_H_ITA];
    o_rate = (int)w[PYST_H_OFF_RATE];
    o_facptr = (int)w[PYST_H_OFF_FACPTR];
    o_fac = (int)w[PYST_H_OFF_FAC];
    o_netptr = (int)w[PYST_H_OFF_NETPTR];
    o_net = (int)w[PYST_H_OFF_NET];
    o_times = (int)w[PYST_H_OFF_TIMES];
    o_out = (int)w[PYST_H_OFF_OUT];
    o_x0 = (int)w[PYST_H_OFF_X0];
    o_spvptr = (int)w[PYST_H_OFF_SPVPTR];
    o_spv = (int)w[PYST_H_OFF_SPV];
    o_g = (int)w[PYST_H_OFF_G];
    o_critptr = (int)w[PYST_H_OFF_CRITPTR];
    o_crit = (int)w[PYST_H_OFF_CRIT];
    o_lawptr = (int)w[PYST_H_OFF_LAWPTR];
    o_law = (int)w[PYST_H_OFF_LAW];
    o_lawc = (int)w[PYST_H_OFF_LAWC];
    nlaw = (int)w[PYST_H_NLAW];
    n_c = (int)w[PYST_H_NC];
    eta = __uint_as_float(w[PYST_H_ETA]);
    const uint64_t tb = (uint64_t)w[PYST_H_TMAX_LO] |
                        ((uint64_t)w[PYST_H_TMAX_HI] << 32);
    t_max = __longlong_as_double((long long)tb);
    pk = nullptr;
    fast = false;
  }
  __device__ __forceinline__ float rate(int j) const {
    return __uint_as_float(w[o_rate + j]);
  }
  __device__ __forceinline__ int facptr(int j) const {
    return (int)w[o_facptr + j];
  }
  __device__ __forceinline__ uint32_t fac(int e) const { return w[o_fac + e]; }
  __device__ __forceinline__ int netptr(int j) const {
    return (int)w[o_netptr + j];
  }
  __device__ __forceinline__ uint32_t net(int e) const { return w[o_net + e]; }
  __device__ __forceinline__ double time(int f) const {
    return (double)__uint_as_float(w[o_times + f]);
  }
  __device__ __forceinline__ int out(int k) const { return (int)w[o_out + k]; }
  __device__ __forceinline__ int x0(int i) const { return (int)w[o_x0 + i]; }
  __device__ __forceinline__ int spvptr(int i) const {
    return (int)w[o_spvptr + i];
  }
  __device__ __forceinline__ uint32_t spv(int e) const { return w[o_spv + e]; }
  __device__ __forceinline__ uint32_t g(int i) const { return w[o_g + i]; }
  __device__ __forceinline__ int critptr(int j) const {
    return (int)w[o_critptr + j];
  }
  __device__ __forceinline__ uint32_t crit(int e) const {
    return w[o_crit + e];
  }
  __device__ __forceinline__ int lawptr(int j) const {
    return (int)w[o_lawptr + j];
  }
  __device__ __forceinline__ uint32_t law(int c) const { return w[o_law + c]; }
  __device__ __forceinline__ double lawc(int k) const {
    return reinterpret_cast<const double*>(w + o_lawc)[k];
  }
};

// entry field decoders
__device__ __forceinline__ int ent_lo(uint32_t e) { return (int)(e & 0xFFFFu); }
__device__ __forceinline__ int ent_hi_s16(uint32_t e) {
  return (int)(int16_t)(uint16_t)(e >> 16);
}
__device__ __forceinline__ int fac_order(uint32_t e) {
  return (int)((e >> 16) & 0xFFu);
}
__device__ __forceinline__ int fac_falling(uint32_t e) {
  return (int)((e >> 24) & 1u);
}

// ------------------------------------------------ bulk-async staging
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar,
                                                      uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

// One bulk copy global -> shared (no multicast).  dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src,
                                         uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after `limit` polls (each try_wait itself blocks
// for a hardware-defined interval), so a lost completion cannot hang.
#define PYST_MBAR_POLL_LIMIT (1 << 22)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          int limit) {
  for (int i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// After a staging wait gave up: wait again, bounded, for the copy still in
// flight, so it cannot land in shared memory that the block has moved on
// from (or released by exiting).
__device__ __forceinline__ bool mbar_drain(uint64_t* bar, uint32_t parity) {
  return mbar_wait(bar, parity, PYST_MBAR_POLL_LIMIT);
}

// Stage `words` (multiple of 4) words of `src` into `dst` with one
// bulk-async copy issued by thread 0; every thread of the block waits on
// phase `parity` of `bar`, for at most `polls` polls (RunArgs.stage_polls).
// Returns false on timeout, the same value in every thread (a block-wide
// vote, so callers may branch on it around barriers); the caller then
// drains the copy (mbar_drain) before reusing or releasing `dst`.  Must be
// called by all threads of the block.  `bar` must have been initialised
// with count 1.
__device__ __forceinline__ bool stage_blob(uint32_t* dst, const uint32_t* src,
                                           int words, uint64_t* bar,
                                           uint32_t parity, int polls) {
  if (threadIdx.x == 0) {
    // Order earlier generic-proxy reads of dst before the async write.
    fence_proxy_async();
    const uint32_t bytes = (uint32_t)words * 4u;
    mbar_arrive_expect_tx(bar, bytes);
    bulk_g2s(dst, src, bytes, bar);
  }
  return __syncthreads_and(mbar_wait(bar, parity, polls)) != 0;
}

}  // namespace pyst
