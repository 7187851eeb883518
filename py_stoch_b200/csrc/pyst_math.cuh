// Counter-based random numbers and deterministic elementary functions.
//
// Every floating-point operation here is an explicitly rounded intrinsic
// (__dadd_rn, __fmul_rn, __fma_rn, ...) and the file is built with
// --fmad=false, so each result is a fixed IEEE-754 function of its inputs.
// A C program doing the same operations in the same order reproduces every
// bit, which is what makes trajectories comparable bit-for-bit with a host
// re-run.
//
// * Philox4x32-10: Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
//   easy as 1, 2, 3", SC'11.  Replaces curand MRG32k3a + curand_init
//   (mod/simulator/simulator.py:62-96): no per-trajectory state array.
// * pyst_log: x = 2^e f, f in [sqrt(1/2), sqrt(2)), log f = 2 atanh(s) with
//   s = (f-1)/(f+1), odd series to s^23 (|s| <= 0.1716, truncation < 1e-17).
// * pyst_exp: x = k ln2 + r, |r| <= ln2/2, Taylor series to r^14.
// * Poisson: inversion by sequential search for lambda < 10; PTRS transformed
//   rejection (W. Hormann, "The transformed rejection method for generating
//   Poisson random variables", Insurance: Mathematics and Economics 12,
//   1993) for lambda >= 10.  Replaces curand_poisson (P1_P2.py:239).
#pragma once
#include <stdint.h>

namespace pyst {

// ---------------------------------------------------------------- Philox
struct Stream {
  uint32_t k0, k1;  // key = seed
  uint32_t c2, c3;  // counter words 2,3 = trajectory id
  uint64_t n;       // block index (counter words 0,1)
};

__device__ __forceinline__ uint4 philox4x32_10(uint32_t c0, uint32_t c1,
                                               uint32_t c2, uint32_t c3,
                                               uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint32_t lo0 = 0xD2511F53u * c0;
    const uint32_t hi0 = __umulhi(0xD2511F53u, c0);
    const uint32_t lo1 = 0xCD9E8D57u * c2;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  return make_uint4(c0, c1, c2, c3);
}

__device__ __forceinline__ Stream make_stream(uint64_t seed, uint64_t id) {
  Stream s;
  s.k0 = (uint32_t)seed;
  s.k1 = (uint32_t)(seed >> 32);
  s.c2 = (uint32_t)id;
  s.c3 = (uint32_t)(id >> 32);
  s.n = 0;
  return s;
}

__device__ __forceinline__ uint4 next_block(Stream& s) {
  const uint4 r = philox4x32_10((uint32_t)s.n, (uint32_t)(s.n >> 32), s.c2,
                                s.c3, s.k0, s.k1);
  s.n++;
  return r;
}

// (0, 1] from 53 bits: hi supplies the top 32, lo the next 21.
__device__ __forceinline__ double u53(uint32_t hi, uint32_t lo) {
  const uint64_t m = ((uint64_t)hi << 21) | (uint64_t)(lo >> 11);
  return (double)(m + 1ull) * 0x1.0p-53;
}
// (0, 1] from the top 24 bits of w.
__device__ __forceinline__ float u24(uint32_t w) {
  return (float)((w >> 8) + 1u) * 0x1.0p-24f;
}
// [0, 1) from all 32 bits of w.
__device__ __forceinline__ double u32co(uint32_t w) {
  return (double)w * 0x1.0p-32;
}

// ------------------------------------------------------- elementary math
#define PYST_LN2_HI 0x1.62e42fee00000p-1
#define PYST_LN2_LO 0x1.a39ef35793c76p-33
#define PYST_INV_LN2 0x1.71547652b82fep+0
#define PYST_HALF_LOG_2PI 0x1.d67f1c864beb4p-1

// Natural log of a positive normal double.
__device__ __forceinline__ double pyst_log(double x) {
  const uint64_t b = (uint64_t)__double_as_longlong(x);
  int e = (int)(b >> 52) - 1023;
  uint64_t mb = (b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;
  if (mb > 0x3FF6A09E667F3BCDull) {
    mb -= 0x0010000000000000ull;
    e += 1;
  }
  const double f = __longlong_as_double((long long)mb);
  const double s = __ddiv_rn(__dsub_rn(f, 1.0), __dadd_rn(f, 1.0));
  const double z = __dmul_rn(s, s);
  double q = 0x1.642c8590b2164p-5;         // 1/23
  q = __fma_rn(q, z, 0x1.8618618618618p-5);  // 1/21
  q = __fma_rn(q, z, 0x1.af286bca1af28p-5);  // 1/19
  q = __fma_rn(q, z, 0x1.e1e1e1e1e1e1ep-5);  // 1/17
  q = __fma_rn(q, z, 0x1.1111111111111p-4);  // 1/15
  q = __fma_rn(q, z, 0x1.3b13b13b13b14p-4);  // 1/13
  q = __fma_rn(q, z, 0x1.745d1745d1746p-4);  // 1/11
  q = __fma_rn(q, z, 0x1.c71c71c71c71cp-4);  // 1/9
  q = __fma_rn(q, z, 0x1.2492492492492p-3);  // 1/7
  q = __fma_rn(q, z, 0x1.999999999999ap-3);  // 1/5
  q = __fma_rn(q, z, 0x1.5555555555555p-2);  // 1/3
  const double s2 = __dmul_rn(2.0, s);
  const double t = __dmul_rn(s2, z);
  const double lf = __fma_rn(t, q, s2);
  const double de = (double)e;
  const double hi = __dmul_rn(de, PYST_LN2_HI);
  const double lo = __fma_rn(de, PYST_LN2_LO, lf);
  return __dadd_rn(hi, lo);
}

// exp(x) for -700 <= x <= 0.
__device__ __forceinline__ double pyst_exp(double x) {
  const double kd = rint(__dmul_rn(x, PYST_INV_LN2));
  const double hi = __fma_rn(-kd, PYST_LN2_HI, x);
  const double r = __fma_rn(-kd, PYST_LN2_LO, hi);
  double p = 0x1.93974a8c07c9dp-37;          // 1/14!
  p = __fma_rn(p, r, 0x1.6124613a86d09p-33);  // 1/13!
  p = __fma_rn(p, r, 0x1.1eed8eff8d898p-29);  // 1/12!
  p = __fma_rn(p, r, 0x1.ae64567f544e4p-26);  // 1/11!
  p = __fma_rn(p, r, 0x1.27e4fb7789f5cp-22);  // 1/10!
  p = __fma_rn(p, r, 0x1.71de3a556c734p-19);  // 1/9!
  p = __fma_rn(p, r, 0x1.a01a01a01a01ap-16);  // 1/8!
  p = __fma_rn(p, r, 0x1.a01a01a01a01ap-13);  // 1/7!
  p = __fma_rn(p, r, 0x1.6c16c16c16c17p-10);  // 1/6!
  p = __fma_rn(p, r, 0x1.1111111111111p-7);   // 1/5!
  p = __fma_rn(p, r, 0x1.5555555555555p-5);   // 1/4!
  p = __fma_rn(p, r, 0x1.5555555555555p-3);   // 1/3!
  p = __fma_rn(p, r, 0.5);
  p = __fma_rn(p, r, 1.0);
  p = __fma_rn(p, r, 1.0);
  const int k = (int)kd;
  const double scale =
      __longlong_as_double((long long)((uint64_t)(k + 1023) << 52));
  return __dmul_rn(p, scale);
}

__device__ __constant__ double c_logfact[16] = {
    0x0.0p+0,
    0x0.0p+0,
    0x1.62e42fefa39efp-1,
    0x1.cab0bfa2a2002p+0,
    0x1.96ca77c922cf9p+1,
    0x1.326643c4479c9p+2,
    0x1.a51273acf01cap+2,
    0x1.10ce1f32dcc30p+3,
    0x1.5358e82fcb70dp+3,
    0x1.99a8921a7f7cfp+3,
    0x1.e357590954d15p+3,
    0x1.180973f3a8d74p+4,
    0x1.3fcba16d50143p+4,
    0x1.68d5a9c3b32cep+4,
    0x1.930f3df162a42p+4,
    0x1.be636a63fd346p+4};

// log(k!) for integral k >= 0: table below 16, Stirling series above.
__device__ __forceinline__ double pyst_logfact(double k) {
  if (k < 16.0) return c_logfact[(int)k];
  const double lnn = pyst_log(k);
  const double inv = __ddiv_rn(1.0, k);
  const double inv2 = __dmul_rn(inv, inv);
  double c = __dmul_rn(inv2, 0x1.a01a01a01a01ap-11);  // 1/1260
  c = __dsub_rn(0x1.6c16c16c16c17p-9, c);             // 1/360
  c = __dmul_rn(inv2, c);
  c = __dsub_rn(0x1.5555555555555p-4, c);             // 1/12
  const double corr = __dmul_rn(inv, c);
  double r = __dmul_rn(__dadd_rn(k, 0.5), lnn);
  r = __dsub_rn(r, k);
  r = __dadd_rn(r, PYST_HALF_LOG_2PI);
  return __dadd_rn(r, corr);
}

#define PYST_POISSON_MAX_LAMBDA 1.0e9f
#define PYST_INVERSION_MAX_K 200
#define PYST_PTRS_MAX_IT 64

// 1/k for k = 1..PYST_INVERSION_MAX_K, correctly rounded (the compiler
// divides at compile time in IEEE double), so the inversion search reads
// the value __drcp_rn((double)k) would compute.
struct PystRcpTable {
  double v[PYST_INVERSION_MAX_K + 1];
  constexpr PystRcpTable() : v() {
    for (int k = 1; k <= PYST_INVERSION_MAX_K; ++k) v[k] = 1.0 / (double)k;
  }
};
__device__ __constant__ PystRcpTable c_rcp = PystRcpTable();

// Counter of the blocks one Poisson draw may use: words (c0, c1 | blk, c2,
// c3) for blk = 0, 1, ... < 32, key (k0, k1).  The leap sampler sets
// c0 = leap index, c1 = 0x80000000 | reaction << 12 | retry << 6, (c2, c3)
// = trajectory id, so every draw has its own counters whatever the order in
// which threads or lanes make them.
struct PoissonKey {
  uint32_t k0, k1, c0, c1, c2, c3;
};

__device__ __forceinline__ uint4 pblock(const PoissonKey& pk, uint32_t blk) {
  return philox4x32_10(pk.c0, pk.c1 | blk, pk.c2, pk.c3, pk.k0, pk.k1);
}

// Poisson(lam) with lam in FP32.  Returns K >= 0; -1 if the rejection
// loop ran out of iterations; -2 if lam is beyond the supported range.
// Draws nothing when lam <= 0.  Kept out of line: a leap calls it once per
// reaction, and one shared copy keeps the instruction footprint small
// (inlined at its one call site of the leap loop it measured 8% slower).
static __device__ __noinline__ int poisson(float lam, const PoissonKey& pk) {
  if (!(lam > 0.0f)) return 0;
  if (!(lam <= PYST_POISSON_MAX_LAMBDA)) return -2;
  if (lam < 10.0f) {
    const uint4 w = pblock(pk, 0u);
    const double u = u32co(w.x);
    const double l = (double)lam;
    double p = pyst_exp(-l);
    double F = p;
    int k = 0;
    while (u > F && k < PYST_INVERSION_MAX_K) {
      k++;
      // p_k = p_{k-1} * lam * (1/k); 1/k correctly rounded
      p = __dmul_rn(__dmul_rn(p, l), c_rcp.v[k]);
      F = __dadd_rn(F, p);
    }
    return k;
  }
  const float slam = __fsqrt_rn(lam);
  const float b = __fadd_rn(0.931f, __fmul_rn(2.53f, slam));
  const float a = __fadd_rn(-0.059f, __fmul_rn(0.02483f, b));
  const float invalpha =
      __fadd_rn(1.1239f, __fdiv_rn(1.1328f, __fsub_rn(b, 3.4f)));
  const float vr = __fsub_rn(0.9277f, __fdiv_rn(3.6224f, __fsub_rn(b, 2.0f)));
  // the two logs of the exact test, computed when a draw first needs it
  // (most draws are accepted by the squeeze above it)
  double loglam = 0.0, log_invalpha = 0.0;
  bool have_logs = false;
  uint4 w = make_uint4(0, 0, 0, 0);
  for (int it = 0; it < PYST_PTRS_MAX_IT; ++it) {
    uint32_t wu, wv;
    if ((it & 1) == 0) {
      w = pblock(pk, (uint32_t)(it >> 1));
      wu = w.x;
      wv = w.y;
    } else {
      wu = w.z;
      wv = w.w;
    }
    const float U = __fsub_rn(u24(wu), 0.5f);
    const float V = u24(wv);
    const float us = __fsub_rn(0.5f, fabsf(U));
    float kf = __fdiv_rn(__fmul_rn(2.0f, a), us);
    kf = __fadd_rn(kf, b);
    kf = __fmul_rn(kf, U);
    kf = __fadd_rn(kf, lam);
    kf = __fadd_rn(kf, 0.43f);
    kf = floorf(kf);
    if (us >= 0.07f && V <= vr) return (int)kf;
    if (kf < 0.0f || (us < 0.013f && V > us)) continue;
    const float den = __fadd_rn(__fdiv_rn(a, __fmul_rn(us, us)), b);
    if (!have_logs) {
      loglam = pyst_log((double)lam);
      log_invalpha = pyst_log((double)invalpha);
      have_logs = true;
    }
    double lhs = __dadd_rn(pyst_log((double)V), log_invalpha);
    lhs = __dsub_rn(lhs, pyst_log((double)den));
    const double kd = (double)kf;
    double rhs = __dadd_rn(-(double)lam, __dmul_rn(kd, loglam));
    rhs = __dsub_rn(rhs, pyst_logfact(kd));
    if (lhs <= rhs) return (int)kf;
  }
  return -1;
}

// FNV-1a style 64-bit mixing of the firing sequence.
#define PYST_FNV_OFFSET 0xcbf29ce484222325ull
#define PYST_FNV_PRIME 0x100000001b3ull
__device__ __forceinline__ uint64_t seq_mix(uint64_t h, uint64_t v) {
  return (h ^ v) * PYST_FNV_PRIME;
}

}  // namespace pyst
