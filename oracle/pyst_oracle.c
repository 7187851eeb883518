/*
 * pyst_oracle.c -- CPU oracle for the B200 stochastic-simulation engine.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests, the smoke
 * test and bench.py's CPU-baseline leg call it; the product never does.
 *
 * It restates the reference's simulation algorithms on the host, one
 * trajectory at a time, with the engine's documented arithmetic (FP32
 * propensities, FP64 clock / total propensity / selection sums, FP32 tau
 * selection and leap sampling) and its Philox4x32-10 stream layout, so
 * that a GPU trajectory and its oracle re-run agree bit for bit:
 *
 *   direct method  mod/simulator/cuGillespie/gillespie.py:70-146
 *                  (+ SaveDynamics 151-162, UpdateState 181-193) and
 *                  mod/simulator/cuTauLeaping/P3.py:71-151
 *   tau-leaping    mod/simulator/cuTauLeaping/P1_P2.py:96-297 with
 *                  DetermineCriticalReactions 299-328, CalculateMuSigma
 *                  330-383, CalculateTau/CalculateG 385-486, critical
 *                  SingleCriticalReaction 488-507, TentativeUpdatedState /
 *                  ValidState 509-540, SaveInterpolatedDynamics 542-584;
 *                  round structure cuTauLeaping.py:49-76
 *
 * Arithmetic is written out operation by operation; build with
 * -ffp-contract=off (no implicit fused multiply-add).  fma() is used only
 * where the engine uses an explicit fused multiply-add.
 *
 * Pinning: Philox4x32-10 is checked against the published known-answer
 * vectors of Salmon et al. (SC'11, Random123 kat_vectors) and, on a GPU,
 * against the CUDA toolkit's curand_Philox4x32_10.  The reference ships no
 * golden trajectories (it has no tests); trajectory-level parity with the
 * reference itself is distribution-level only (its curand MRG32k3a stream
 * cannot be reproduced), so trajectory parity with the reference is
 * unpinned; the oracle is checked against exact moments of first-order
 * networks instead.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <pthread.h>
#include <unistd.h>

/* ------------------------------------------------------------ Philox */

void oracle_philox(const uint32_t ctr[4], const uint32_t key[2],
                   uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

typedef struct {
  uint32_t k0, k1, c2, c3;
  uint64_t n;
} ostream;

static void os_block(ostream* s, uint32_t w[4]) {
  uint32_t ctr[4] = {(uint32_t)s->n, (uint32_t)(s->n >> 32), s->c2, s->c3};
  uint32_t key[2] = {s->k0, s->k1};
  oracle_philox(ctr, key, w);
  s->n++;
}

static double u53(uint32_t hi, uint32_t lo) {
  uint64_t m = ((uint64_t)hi << 21) | (uint64_t)(lo >> 11);
  return (double)(m + 1ull) * 0x1.0p-53;
}
static float u24(uint32_t w) { return (float)((w >> 8) + 1u) * 0x1.0p-24f; }
static double u32co(uint32_t w) { return (double)w * 0x1.0p-32; }

/* ------------------------------------------------- elementary math */

#define LN2_HI 0x1.62e42fee00000p-1
#define LN2_LO 0x1.a39ef35793c76p-33
#define INV_LN2 0x1.71547652b82fep+0
#define HALF_LOG_2PI 0x1.d67f1c864beb4p-1

double oracle_log(double x) {
  uint64_t b;
  memcpy(&b, &x, 8);
  int e = (int)(b >> 52) - 1023;
  uint64_t mb = (b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;
  if (mb > 0x3FF6A09E667F3BCDull) {
    mb -= 0x0010000000000000ull;
    e += 1;
  }
  double f;
  memcpy(&f, &mb, 8);
  double num = f - 1.0;
  double den = f + 1.0;
  double s = num / den;
  double z = s * s;
  double q = 0x1.642c8590b2164p-5;
  q = fma(q, z, 0x1.8618618618618p-5);
  q = fma(q, z, 0x1.af286bca1af28p-5);
  q = fma(q, z, 0x1.e1e1e1e1e1e1ep-5);
  q = fma(q, z, 0x1.1111111111111p-4);
  q = fma(q, z, 0x1.3b13b13b13b14p-4);
  q = fma(q, z, 0x1.745d1745d1746p-4);
  q = fma(q, z, 0x1.c71c71c71c71cp-4);
  q = fma(q, z, 0x1.2492492492492p-3);
  q = fma(q, z, 0x1.999999999999ap-3);
  q = fma(q, z, 0x1.5555555555555p-2);
  double s2 = 2.0 * s;
  double t = s2 * z;
  double lf = fma(t, q, s2);
  double de = (double)e;
  double hi = de * LN2_HI;
  double lo = fma(de, LN2_LO, lf);
  return hi + lo;
}

double oracle_exp(double x) {
  double kd = rint(x * INV_LN2);
  double hi = fma(-kd, LN2_HI, x);
  double r = fma(-kd, LN2_LO, hi);
  double p = 0x1.93974a8c07c9dp-37;
  p = fma(p, r, 0x1.6124613a86d09p-33);
  p = fma(p, r, 0x1.1eed8eff8d898p-29);
  p = fma(p, r, 0x1.ae64567f544e4p-26);
  p = fma(p, r, 0x1.27e4fb7789f5cp-22);
  p = fma(p, r, 0x1.71de3a556c734p-19);
  p = fma(p, r, 0x1.a01a01a01a01ap-16);
  p = fma(p, r, 0x1.a01a01a01a01ap-13);
  p = fma(p, r, 0x1.6c16c16c16c17p-10);
  p = fma(p, r, 0x1.1111111111111p-7);
  p = fma(p, r, 0x1.5555555555555p-5);
  p = fma(p, r, 0x1.5555555555555p-3);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  int k = (int)kd;
  uint64_t sb = (uint64_t)(k + 1023) << 52;
  double scale;
  memcpy(&scale, &sb, 8);
  return p * scale;
}

static const double LOGFACT[16] = {
    0x0.0p+0,           0x0.0p+0,           0x1.62e42fefa39efp-1,
    0x1.cab0bfa2a2002p+0, 0x1.96ca77c922cf9p+1, 0x1.326643c4479c9p+2,
    0x1.a51273acf01cap+2, 0x1.10ce1f32dcc30p+3, 0x1.5358e82fcb70dp+3,
    0x1.99a8921a7f7cfp+3, 0x1.e357590954d15p+3, 0x1.180973f3a8d74p+4,
    0x1.3fcba16d50143p+4, 0x1.68d5a9c3b32cep+4, 0x1.930f3df162a42p+4,
    0x1.be636a63fd346p+4};

double oracle_logfact(double k) {
  if (k < 16.0) return LOGFACT[(int)k];
  double lnn = oracle_log(k);
  double inv = 1.0 / k;
  double inv2 = inv * inv;
  double c = inv2 * 0x1.a01a01a01a01ap-11;
  c = 0x1.6c16c16c16c17p-9 - c;
  c = inv2 * c;
  c = 0x1.5555555555555p-4 - c;
  double corr = inv * c;
  double r = (k + 0.5) * lnn;
  r = r - k;
  r = r + HALF_LOG_2PI;
  return r + corr;
}

/* Poisson with the block counter (c0, c1 | blk, c2, c3). */
typedef struct {
  uint32_t k0, k1, c0, c1, c2, c3;
} opkey;

static void pblock(const opkey* pk, uint32_t blk, uint32_t w[4]) {
  uint32_t ctr[4] = {pk->c0, pk->c1 | blk, pk->c2, pk->c3};
  uint32_t key[2] = {pk->k0, pk->k1};
  oracle_philox(ctr, key, w);
}

/* cnt (optional): [0] inversion draws, [1] inversion search iterations,
 * [2] PTRS draws, [3] PTRS iterations. */
static int oracle_poisson_counted(float lam, const opkey* pk, int64_t* cnt) {
  if (!(lam > 0.0f)) return 0;
  if (!(lam <= 1.0e9f)) return -2;
  uint32_t w[4];
  if (lam < 10.0f) {
    if (cnt) cnt[0]++;
    pblock(pk, 0u, w);
    double u = u32co(w[0]);
    double l = (double)lam;
    double p = oracle_exp(-l);
    double F = p;
    int k = 0;
    while (u > F && k < 200) {
      k++;
      if (cnt) cnt[1]++;
      double inv = 1.0 / (double)k;
      p = (p * l) * inv;
      F = F + p;
    }
    return k;
  }
  float slam = sqrtf(lam);
  double loglam = oracle_log((double)lam);
  float b = 0.931f + 2.53f * slam;
  float a = -0.059f + 0.02483f * b;
  float invalpha = 1.1239f + 1.1328f / (b - 3.4f);
  float vr = 0.9277f - 3.6224f / (b - 2.0f);
  double log_invalpha = oracle_log((double)invalpha);
  if (cnt) cnt[2]++;
  for (int it = 0; it < 64; ++it) {
    uint32_t wu, wv;
    if (cnt) cnt[3]++;
    if ((it & 1) == 0) {
      pblock(pk, (uint32_t)(it >> 1), w);
      wu = w[0];
      wv = w[1];
    } else {
      wu = w[2];
      wv = w[3];
    }
    float U = u24(wu) - 0.5f;
    float V = u24(wv);
    float us = 0.5f - fabsf(U);
    float kf = (2.0f * a) / us;
    kf = kf + b;
    kf = kf * U;
    kf = kf + lam;
    kf = kf + 0.43f;
    kf = floorf(kf);
    if (us >= 0.07f && V <= vr) return (int)kf;
    if (kf < 0.0f || (us < 0.013f && V > us)) continue;
    float den = a / (us * us) + b;
    double lhs = oracle_log((double)V) + log_invalpha;
    lhs = lhs - oracle_log((double)den);
    double kd = (double)kf;
    double rhs = -(double)lam + kd * loglam;
    rhs = rhs - oracle_logfact(kd);
    if (lhs <= rhs) return (int)kf;
  }
  return -1;
}

int oracle_poisson(float lam, const opkey* pk) {
  return oracle_poisson_counted(lam, pk, NULL);
}

/* ------------------------------------------------------------- model */

typedef struct {
  int S, R, kappa, ita;
  const int32_t* order;     /* [S*R] */
  const uint8_t* falling;   /* [S*R] */
  const int32_t* pre;       /* [S*R] */
  const int32_t* net;       /* [S*R] */
  const double* rate;       /* [R] (rounded to FP32 here) */
  const int32_t* x0;        /* [S] */
  const int32_t* hor;       /* [S] */
  const int32_t* hor_type;  /* [S] */
  const float* times;       /* [ita] */
  const int32_t* out;       /* [kappa] */
  float eta;
  int n_c;
  /* general kinetic laws (kinetic.py; engine eval_law): NULL = none */
  const int32_t* law_ptr;   /* [R+1] */
  const uint32_t* law_code;
  const double* law_const;
} omodel;

typedef struct {
  uint64_t seed;
  int64_t id_base;
  int method;   /* 0 direct, 1 tau */
  int warp;     /* 0 sequential sums, 1 32-lane slice sums + scan */
  int ssa_fallback;
  int max_retries;
  int64_t step_budget;
} orun;

typedef struct {
  int32_t* samples; /* [kappa][ita][n] */
  int64_t n;
  uint8_t* status;
  int64_t* events;
  uint64_t* seqhash;
  double* t_final;
  double* score; /* [n][R] */
  int64_t* steps; /* [n][6] (optional): SSA steps, leaps, inversion Poisson
                     draws, their search iterations, PTRS draws, their
                     iterations */
} oout;

#define FNV_OFF 0xcbf29ce484222325ull
#define FNV_PRIME 0x100000001b3ull
static uint64_t mix(uint64_t h, uint64_t v) { return (h ^ v) * FNV_PRIME; }

/* Kinetic-law programs (py_stoch_b200/kinetic.py), evaluated in FP64 one
 * rounded operation at a time like the engine's eval_law
 * (py_stoch_b200/csrc/pyst_engine.cuh). */
static double law_idiv(double a, double b) {
  if (b == 0.0) return NAN;
  double q = trunc(a / b);
  double rem = fma(-q, b, a);
  if (q != 0.0 && rem != 0.0 && ((rem < 0.0) != (a < 0.0)))
    q = q - copysign(1.0, q);
  return q;
}

static double law_exp(double a) {
  if (!(a == a)) return a;
  if (a > 709.0) return INFINITY;
  if (a < -708.0) return 0.0;
  return oracle_exp(a);
}

static double law_ln(double a) {
  if (!(a >= 0.0)) return NAN;
  if (a == 0.0) return -INFINITY;
  if (a > 1.7976931348623157e308) return a;
  return oracle_log(a);
}

static float eval_law(const omodel* m, int j, const int32_t* x) {
  double st[8];
  int sp = 0;
  for (int c = m->law_ptr[j]; c < m->law_ptr[j + 1]; ++c) {
    uint32_t wd = m->law_code[c];
    int op = (int)(wd >> 24), arg = (int)(wd & 0xFFFFFFu);
    if (op == 1 || op == 2 || op == 16) {
      if (sp >= 8 || (op == 16 && sp < 1)) return NAN;
      st[sp] = op == 1 ? (double)x[arg]
                       : (op == 2 ? m->law_const[arg] : st[sp - 1]);
      ++sp;
    } else if (op >= 3 && op <= 7) {
      if (sp < 2) return NAN;
      double b = st[--sp], a = st[sp - 1], r;
      if (op == 3) r = a + b;
      else if (op == 4) r = a - b;
      else if (op == 5) r = a * b;
      else if (op == 6) r = a / b;
      else r = law_idiv(a, b);
      st[sp - 1] = r;
    } else {
      if (sp < 1) return NAN;
      double a = st[sp - 1], r;
      if (op == 8) r = -a;
      else if (op == 10) r = law_exp(a);
      else if (op == 11) r = law_ln(a);
      else if (op == 12) r = sqrt(a);
      else if (op == 13) r = fabs(a);
      else if (op == 14) r = floor(a);
      else if (op == 15) r = ceil(a);
      else return NAN;
      st[sp - 1] = r;
    }
  }
  return sp == 1 ? (float)st[0] : NAN;
}

static int has_law(const omodel* m, int j) {
  return m->law_ptr && m->law_ptr[j + 1] > m->law_ptr[j];
}

static int valid_rate(float a) { return a >= 0.0f && a <= 3.4028234663852886e38f; }

/* Propensity of reaction j: the reaction's kinetic-law program, or the
 * FP32 product, species ascending, factor index ascending. */
static float prop(const omodel* m, const float* rate32, int j,
                  const int32_t* x) {
  if (has_law(m, j)) return eval_law(m, j, x);
  float a = rate32[j];
  for (int i = 0; i < m->S; ++i) {
    int n = m->order[(size_t)i * m->R + j];
    if (n <= 0) continue;
    int fall = m->falling ? (m->falling[(size_t)i * m->R + j] ? 1 : 0) : 1;
    for (int q = 0; q < n; ++q) a = a * (float)(x[i] - q * fall);
  }
  return a;
}

static float gfun(int H, int Ht, int x) {
  float xf = (float)x;
  if (H == 1) return 1.0f;
  if (H == 2) {
    if (Ht == 2) return 2.0f + 1.0f / (xf - 1.0f);
    return 2.0f;
  }
  if (H == 3) {
    if (Ht == 3) {
      float t1 = 1.0f / (xf - 1.0f);
      float t2 = 2.0f / (xf - 2.0f);
      return (3.0f + t1) + t2;
    }
    if (Ht == 2) return 1.5f * (2.0f + 1.0f / (xf - 1.0f));
    return 3.0f;
  }
  if (H >= 4) {
    /* Cao's g generalised past third order: (H/n)(n + sum k/(x-k)) */
    int n = Ht < 1 ? 1 : Ht;
    float sm = (float)n;
    for (int k = 1; k < n; ++k) sm = sm + (float)k / (xf - (float)k);
    return ((float)H / (float)n) * sm;
  }
  return 0.0f;
}

/* Kogge-Stone inclusive scan of 32 lane values, in the warp's order. */
static void scan32(const double* part, double* incl) {
  double v[32], nv[32];
  for (int l = 0; l < 32; ++l) v[l] = part[l];
  for (int d = 1; d < 32; d <<= 1) {
    for (int l = 0; l < 32; ++l) nv[l] = (l >= d) ? (v[l - d] + v[l]) : v[l];
    for (int l = 0; l < 32; ++l) v[l] = nv[l];
  }
  for (int l = 0; l < 32; ++l) incl[l] = v[l];
}

/* total of the a_j with mask (NULL = all), in the mapping's order */
static double total(const orun* ru, int R, const float* a,
                    const uint8_t* mask, double* part, double* incl) {
  if (!ru->warp) {
    double s = 0.0;
    for (int j = 0; j < R; ++j)
      if (!mask || mask[j]) s = s + (double)a[j];
    return s;
  }
  int c = (R + 31) >> 5;
  for (int l = 0; l < 32; ++l) {
    int j0 = l * c < R ? l * c : R;
    int j1 = j0 + c < R ? j0 + c : R;
    double p = 0.0;
    for (int j = j0; j < j1; ++j)
      if (!mask || mask[j]) p = p + (double)a[j];
    part[l] = p;
  }
  scan32(part, incl);
  return incl[31];
}

/* first reaction whose cumulative sum reaches r */
static int select_rx(const orun* ru, int R, const float* a,
                     const uint8_t* mask, double r, const double* part,
                     const double* incl) {
  if (!ru->warp) {
    double cum = 0.0;
    int lastnz = -1;
    for (int j = 0; j < R; ++j) {
      if (mask && !mask[j]) continue;
      cum = cum + (double)a[j];
      if (a[j] > 0.0f) lastnz = j;
      if (cum >= r) return j;
    }
    return lastnz;
  }
  int c = (R + 31) >> 5;
  int L = -1, lastp = -1;
  for (int l = 0; l < 32; ++l) {
    if (part[l] > 0.0) {
      lastp = l;
      if (L < 0 && incl[l] >= r) L = l;
    }
  }
  if (L < 0) L = lastp;
  int j0 = L * c < R ? L * c : R;
  int j1 = j0 + c < R ? j0 + c : R;
  double rr = r - (incl[L] - part[L]);
  double cum = 0.0;
  int lastnz = -1;
  for (int j = j0; j < j1; ++j) {
    if (mask && !mask[j]) continue;
    cum = cum + (double)a[j];
    if (a[j] > 0.0f) lastnz = j;
    if (cum >= rr) return j;
  }
  return lastnz;
}

static void store(const omodel* m, const oout* o, int64_t u, int k, int f,
                  int32_t v) {
  o->samples[((int64_t)k * m->ita + f) * o->n + u] = v;
}

#define I32MAX 2147483647ll

static void one_trajectory(const omodel* m, const float* rate32,
                           const orun* ru, const oout* o, int64_t u,
                           float* a, uint8_t* crit, int32_t* x, int64_t* dx,
                           float* mu, float* s2, int32_t* K, double* integ,
                           double* cnt) {
  const int S = m->S, R = m->R, ita = m->ita, kappa = m->kappa;
  double part[32], incl[32], partc[32], inclc[32];
  uint64_t id = (uint64_t)(ru->id_base + u);
  ostream rs = {(uint32_t)ru->seed, (uint32_t)(ru->seed >> 32), (uint32_t)id,
                (uint32_t)(id >> 32), 0};
  for (int i = 0; i < S; ++i) x[i] = m->x0[i];
  for (int j = 0; j < R; ++j) {
    integ[j] = 0.0;
    cnt[j] = 0.0;
  }
  double t = 0.0;
  int f = 0;
  int64_t events = 0, steps = 0, n_ssa = 0, n_leap = 0;
  int64_t pcnt[4] = {0, 0, 0, 0};
  uint64_t h = FNV_OFF;
  int status = 0, fill_state = 0;
  int64_t budget = ru->step_budget ? ru->step_budget : (1ll << 62);
  double t_end = (double)m->times[ita - 1];
  int ssa_mode = ru->method == 0;
  int ssa_left = 0;
  uint32_t leap_q = 0;

  for (;;) {
    int bad_rate = 0;
    for (int j = 0; j < R; ++j) {
      a[j] = prop(m, rate32, j, x);
      if (m->law_ptr && !valid_rate(a[j])) bad_rate = 1;
    }
    if (bad_rate) {
      status = 7;
      break;
    }
    double a0 = total(ru, R, a, NULL, part, incl);
    if (a0 == 0.0) {
      status = 1;
      fill_state = 1;
      break;
    }
    if (steps >= budget) {
      status = 2;
      break;
    }
    if (ru->method == 1 && !ssa_mode) {
      /* DetermineCriticalReactions: net change v < 0 and |v| n_c > x */
      for (int j = 0; j < R; ++j) {
        crit[j] = 0;
        for (int i = 0; i < S; ++i) {
          int v = m->net[(size_t)i * R + j];
          if (v < 0 && (int64_t)(-v) * m->n_c > (int64_t)x[i]) crit[j] = 1;
        }
      }
      /* CalculateMuSigma + CalculateTau, species-major, j ascending */
      float tau1 = INFINITY;
      for (int i = 0; i < S; ++i) {
        int reactant = 0;
        for (int j = 0; j < R; ++j)
          if (m->pre[(size_t)i * R + j] > 0) reactant = 1;
        if (!reactant) continue;
        float mui = 0.0f, s2i = 0.0f;
        for (int j = 0; j < R; ++j) {
          int v = m->net[(size_t)i * R + j];
          if (v == 0 || crit[j]) continue;
          mui = mui + (float)v * a[j];
          s2i = s2i + (float)(v * v) * a[j];
        }
        float g = gfun(m->hor ? m->hor[i] : 0, m->hor_type ? m->hor_type[i] : 0,
                       x[i]);
        float num = fmaxf((m->eta * (float)x[i]) / g, 1.0f);
        float lhs = num / fabsf(mui);
        float rhs = (num * num) / s2i;
        float cnd = fminf(lhs, rhs);
        if (cnd < tau1) tau1 = cnd;
      }
      if ((double)tau1 < 10.0 / a0) {
        ssa_mode = 1;
        ssa_left = ru->ssa_fallback;
        /* fall through to one SSA step with the same propensities */
      } else {
        steps++;
        n_leap++;
        double a0c = total(ru, R, a, crit, partc, inclc);
        double tau2 = INFINITY;
        uint32_t wc[4] = {0, 0, 0, 0};
        if (a0c > 0.0) {
          os_block(&rs, wc);
          tau2 = -oracle_log(u53(wc[0], wc[1])) / a0c;
        }
        double tau1d = (double)tau1;
        double tau = (tau2 < tau1d) ? tau2 : tau1d;
        int kcrit = -1;
        if (tau1d > tau2) {
          double r = u53(wc[2], wc[3]) * a0c;
          kcrit = select_rx(ru, R, a, crit, r, partc, inclc);
        }
        int retry = 0, ok = 0;
        for (;;) {
          int bad = 0;
          for (int j = 0; j < R; ++j) {
            if (crit[j]) {
              K[j] = (j == kcrit) ? 1 : 0;
            } else {
              float lam = a[j] * (float)tau;
              opkey pk = {rs.k0, rs.k1, leap_q,
                          0x80000000u | ((uint32_t)j << 12) |
                              ((uint32_t)retry << 6),
                          rs.c2, rs.c3};
              int k = oracle_poisson_counted(lam, &pk, pcnt);
              if (k < 0) bad = 1;
              K[j] = k < 0 ? 0 : k;
            }
          }
          if (bad) {
            status = 5;
            break;
          }
          int neg = 0, over = 0;
          for (int i = 0; i < S; ++i) {
            int64_t d = 0;
            for (int j = 0; j < R; ++j)
              d += (int64_t)K[j] * m->net[(size_t)i * R + j];
            dx[i] = d;
            int64_t nx = (int64_t)x[i] + d;
            if (nx < 0) neg = 1;
            if (nx > I32MAX) over = 1;
          }
          if (over) {
            status = 3;
            break;
          }
          if (!neg) {
            ok = 1;
            break;
          }
          tau = tau * 0.5;
          retry++;
          if (retry > ru->max_retries) {
            status = 4;
            break;
          }
        }
        if (!ok) break;
        leap_q++;
        double tn = t + tau;
        int64_t fired = 0;
        h = mix(h, 0xFFFFFFFFull);
        for (int j = 0; j < R; ++j) {
          fired += K[j];
          if (K[j] != 0) h = mix(h, ((uint64_t)j << 32) | (uint32_t)K[j]);
          cnt[j] = cnt[j] + (double)K[j];
          integ[j] = integ[j] + (double)a[j] * tau;
        }
        int done = 0;
        while (tn >= (double)m->times[f]) {
          double frac = ((double)m->times[f] - t) / tau;
          for (int k = 0; k < kappa; ++k) {
            int i = m->out[k];
            double inc = rint((double)dx[i] * frac);
            store(m, o, u, k, f, x[i] + (int)inc);
          }
          f++;
          if (f == ita) {
            done = 1;
            break;
          }
        }
        for (int i = 0; i < S; ++i) x[i] = (int32_t)((int64_t)x[i] + dx[i]);
        events += fired;
        t = tn;
        if (done) break;
        continue;
      }
    }
    /* one direct-method step */
    steps++;
    n_ssa++;
    uint32_t w[4];
    os_block(&rs, w);
    double tau = -oracle_log(u53(w[0], w[1])) / a0;
    double r = u53(w[2], w[3]) * a0;
    int sel = select_rx(ru, R, a, NULL, r, part, incl);
    double tn = t + tau;
    double dt = (tn >= t_end) ? (t_end - t) : tau;
    for (int j = 0; j < R; ++j) integ[j] = integ[j] + (double)a[j] * dt;
    int done = 0;
    while (tn >= (double)m->times[f]) {
      for (int k = 0; k < kappa; ++k) store(m, o, u, k, f, x[m->out[k]]);
      f++;
      if (f == ita) {
        done = 1;
        break;
      }
    }
    t = tn;
    if (done) break;
    int over = 0;
    for (int i = 0; i < S; ++i) {
      int v = m->net[(size_t)i * R + sel];
      if (v == 0) continue;
      int64_t nx = (int64_t)x[i] + v;
      if (nx < 0 || nx > I32MAX) over = 1;
      else x[i] = (int32_t)nx;
    }
    if (over) {
      status = 3;
      break;
    }
    events++;
    h = mix(h, (uint64_t)sel);
    cnt[sel] = cnt[sel] + 1.0;
    if (ru->method == 1) {
      if (--ssa_left <= 0) ssa_mode = 0;
    }
  }
  for (; f < ita; ++f)
    for (int k = 0; k < kappa; ++k)
      store(m, o, u, k, f, fill_state ? x[m->out[k]] : -1);
  if (o->status) o->status[u] = (uint8_t)status;
  if (o->events) o->events[u] = events;
  if (o->seqhash) o->seqhash[u] = h;
  if (o->t_final) o->t_final[u] = t;
  if (o->steps) {
    o->steps[6 * u] = n_ssa;
    o->steps[6 * u + 1] = n_leap;
    for (int q = 0; q < 4; ++q) o->steps[6 * u + 2 + q] = pcnt[q];
  }
  if (o->score)
    for (int j = 0; j < R; ++j) o->score[u * R + j] = cnt[j] - integ[j];
}

typedef struct {
  const omodel* m;
  const float* rate32;
  const orun* ru;
  const oout* o;
  int64_t u1;
  int64_t next; /* shared work counter */
  pthread_mutex_t lock;
  int err;
} ojob;

static void* worker(void* arg) {
  ojob* jb = (ojob*)arg;
  const int S = jb->m->S, R = jb->m->R;
  float* a = (float*)malloc(sizeof(float) * R);
  uint8_t* crit = (uint8_t*)malloc((size_t)R);
  int32_t* x = (int32_t*)malloc(sizeof(int32_t) * S);
  int64_t* dx = (int64_t*)malloc(sizeof(int64_t) * S);
  float* mu = (float*)malloc(sizeof(float) * S);
  float* s2 = (float*)malloc(sizeof(float) * S);
  int32_t* K = (int32_t*)malloc(sizeof(int32_t) * R);
  double* integ = (double*)malloc(sizeof(double) * R);
  double* cnt = (double*)malloc(sizeof(double) * R);
  if (!a || !crit || !x || !dx || !mu || !s2 || !K || !integ || !cnt) {
    pthread_mutex_lock(&jb->lock);
    jb->err = 2;
    pthread_mutex_unlock(&jb->lock);
  } else {
    for (;;) {
      pthread_mutex_lock(&jb->lock);
      int64_t u = jb->next++;
      pthread_mutex_unlock(&jb->lock);
      if (u >= jb->u1) break;
      one_trajectory(jb->m, jb->rate32, jb->ru, jb->o, u, a, crit, x, dx, mu,
                     s2, K, integ, cnt);
    }
  }
  free(a);
  free(crit);
  free(x);
  free(dx);
  free(mu);
  free(s2);
  free(K);
  free(integ);
  free(cnt);
  return NULL;
}

int oracle_max_threads(void) {
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 1;
}

/* Simulate trajectories [u0, u1) of the run on nthreads host threads
 * (<= 0: one per online core).  Results do not depend on nthreads. */
int oracle_simulate(const omodel* m, const orun* ru, const oout* o, int64_t u0,
                    int64_t u1, int nthreads) {
  if (!m || !ru || !o || m->S < 1 || m->R < 1) return 1;
  float* rate32 = (float*)malloc(sizeof(float) * m->R);
  if (!rate32) return 2;
  for (int j = 0; j < m->R; ++j) rate32[j] = (float)m->rate[j];
  if (nthreads <= 0) nthreads = oracle_max_threads();
  if (nthreads > 256) nthreads = 256;
  ojob jb;
  jb.m = m;
  jb.rate32 = rate32;
  jb.ru = ru;
  jb.o = o;
  jb.u1 = u1;
  jb.next = u0;
  jb.err = 0;
  pthread_mutex_init(&jb.lock, NULL);
  pthread_t th[256];
  int started = 0;
  for (int i = 1; i < nthreads; ++i)
    if (pthread_create(&th[started], NULL, worker, &jb) == 0) started++;
  worker(&jb);
  for (int i = 0; i < started; ++i) pthread_join(th[i], NULL);
  pthread_mutex_destroy(&jb.lock);
  free(rate32);
  return jb.err;
}

/* batch helpers for tests: vectorised math and Poisson draws */
void oracle_math(const double* x, int64_t n, int which, double* out) {
  for (int64_t i = 0; i < n; ++i) {
    if (which == 0) out[i] = oracle_log(x[i]);
    else if (which == 1) out[i] = oracle_exp(x[i]);
    else out[i] = oracle_logfact(x[i]);
  }
}

/* Same stream layout as the engine's test hook: trajectory id i, leap
 * index 7, reaction i mod 1024, retry 3. */
void oracle_poisson_batch(const float* lam, int64_t n, uint64_t seed,
                          int32_t* out) {
  for (int64_t i = 0; i < n; ++i) {
    uint64_t id = (uint64_t)i;
    opkey pk = {(uint32_t)seed, (uint32_t)(seed >> 32), 7u,
                0x80000000u | ((uint32_t)(i & 1023) << 12) | (3u << 6),
                (uint32_t)id, (uint32_t)(id >> 32)};
    out[i] = oracle_poisson(lam[i], &pk);
  }
}

void oracle_philox_stream(uint64_t seed, uint64_t id, uint64_t n0,
                          int64_t count, uint32_t* out) {
  for (int64_t i = 0; i < count; ++i) {
    ostream s = {(uint32_t)seed, (uint32_t)(seed >> 32), (uint32_t)id,
                 (uint32_t)(id >> 32), n0 + (uint64_t)i};
    os_block(&s, out + 4 * i);
  }
}
