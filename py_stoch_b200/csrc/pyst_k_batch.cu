// Batched persistent kernel: many models of uneven size in one launch.
// Blocks take work items (one model, its trajectories and output offsets)
// from a device queue (an atomic counter in caller workspace), stage the
// item's model blob into shared memory with one bulk-async copy, and run its
// trajectories thread-per-trajectory or warp-per-trajectory as the item
// says.  Replaces the reference's one-JIT-and-launch-sequence-per-model
// sweep (examples/*_sim.py loops over CuTauLeaping().run, e.g.
// examples/schlogl_sim.py:66-80).  Built once per PYST_SCORE flavour.
#include "pyst_launch.cuh"

// Blocks of 128 threads per SM the register allocation must allow: 6 (at
// most 80 registers) measured 11% faster than no bound on the
// Schlogl/Lotka-Volterra sweep (2048 models, scores, statistics) and 1.5%
// slower on synthetic networks of up to 256 reactions; 0 leaves it open.
#ifndef PYST_BATCH_MINB
#define PYST_BATCH_MINB 6
#endif
#if PYST_BATCH_MINB > 0
#define PYST_BATCH_BOUNDS __launch_bounds__(128, PYST_BATCH_MINB)
#else
#define PYST_BATCH_BOUNDS __launch_bounds__(128)
#endif

namespace pyst {
// nvcc gives template functions of an anonymous namespace weak external
// linkage on the host side, so the flavours built from this file would be
// merged at link time; a per-flavour namespace keeps them apart.
namespace PYST_CAT(batch_flavour_, PYST_SCORE, ) {

// Summary statistics and score Jacobians of one finished model (U
// trajectories), computed by the block that ran it -- or, for a model split
// into chunks, ran its last chunk -- from the samples (and scores) written
// for it, sums over trajectories in trajectory order.  Loads bypass L1
// (other blocks wrote part of the data).  Means and variances go to shared
// scratch `ms` when 2*kappa*ita doubles fit, else they are recomputed.
__device__ void item_epilogue(const ModelView& m, const pyst_batch_item& item,
                              int64_t U, const OutBase& ob, double* ms,
                              int ms_bytes) {
  const int ita = m.ita, KF = m.kappa * m.ita, R = m.R;
  if (U <= 0) return;
  const int32_t* smp = ob.samples + item.sample_offset;
  const double dU = (double)U;
  const bool keep = (size_t)KF * 16 <= (size_t)ms_bytes;
  auto row_moments = [&](int kf, double& mean, double& var) {
    const int32_t* row = smp + (int64_t)kf * U;
    double s = 0.0, s2 = 0.0;
    for (int64_t u = 0; u < U; ++u) {
      const double x = (double)__ldcg(row + u);
      s = __dadd_rn(s, x);
      s2 = __dadd_rn(s2, __dmul_rn(x, x));
    }
    mean = __ddiv_rn(s, dU);
    var = __dsub_rn(__ddiv_rn(s2, dU), __dmul_rn(mean, mean));
  };
  for (int kf = threadIdx.x; kf < KF; kf += blockDim.x) {
    double mean, var;
    row_moments(kf, mean, var);
    if (keep) {
      ms[2 * kf] = mean;
      ms[2 * kf + 1] = var;
    }
    if (ob.stats) {
      double corr = 0.0;
      const int f = kf % ita;
      if (f + 1 < ita) {
        double mb, vb;
        row_moments(kf + 1, mb, vb);
        const int32_t* ra_ = smp + (int64_t)kf * U;
        const int32_t* rb = ra_ + U;
        double sab = 0.0;
        for (int64_t u = 0; u < U; ++u)
          sab = __dadd_rn(sab, __dmul_rn((double)__ldcg(ra_ + u),
                                         (double)__ldcg(rb + u)));
        const double cov = __dsub_rn(__ddiv_rn(sab, dU), __dmul_rn(mean, mb));
        const double den = __dmul_rn(var, vb);
        if (den > 0.0) corr = __ddiv_rn(cov, __dsqrt_rn(den));
      }
      double* o = ob.stats + item.stats_offset + (int64_t)kf * 3;
      o[0] = mean;
      o[1] = var;
      o[2] = corr;
    }
  }
  if (!ob.jac || !ob.score) return;
  __syncthreads();
  const double* sc = ob.score + item.score_offset;
  for (int idx = threadIdx.x; idx < KF * R; idx += blockDim.x) {
    const int kf = idx / R, j = idx - kf * R;
    double mean, var;
    if (keep) {
      mean = ms[2 * kf];
      var = ms[2 * kf + 1];
    } else {
      row_moments(kf, mean, var);
    }
    const int32_t* row = smp + (int64_t)kf * U;
    double gm = 0.0, gv = 0.0;
    for (int64_t u = 0; u < U; ++u) {
      const double d = __dsub_rn((double)__ldcg(row + u), mean);
      const double s = __ldcg(sc + u * R + j);
      gm = __dadd_rn(gm, __dmul_rn(d, s));
      gv = __dadd_rn(gv, __dmul_rn(__dsub_rn(__dmul_rn(d, d), var), s));
    }
    double* o = ob.jac + item.jac_offset;
    o[(int64_t)kf * R + j] = __ddiv_rn(gm, dU);
    o[((int64_t)KF + kf) * R + j] = __ddiv_rn(gv, dU);
  }
}

template <bool SCORE>
__global__ void PYST_BATCH_BOUNDS
    k_batch(const uint32_t* __restrict__ gblobs,
            const pyst_batch_item* __restrict__ items, int64_t n_items,
            RunArgs ra, OutBase ob, unsigned long long* queue, unsigned* done,
            int max_blob_words, int warp_bytes, int dyn_bytes, int pk_bytes) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long s_item;
  __shared__ int s_last;
  uint32_t* sblob = (uint32_t*)smem;
  uint64_t* bar = (uint64_t*)(smem + (size_t)max_blob_words * 4);
  // packed reaction descriptors of the current item (thread mapping)
  uint32_t* spk = (uint32_t*)(smem + (size_t)max_blob_words * 4 + 16);
  unsigned char* dyn =
      smem + (size_t)max_blob_words * 4 + 16 + (size_t)pk_bytes;
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_barrier_init();
  }
  __syncthreads();
  const int bs = blockDim.x, nw = bs >> 5, wid = threadIdx.x >> 5;
  uint32_t parity = 0;
  while (true) {
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(queue, 1ull);
    __syncthreads();
    const long long it = s_item;
    if (it >= n_items) break;
    const pyst_batch_item item = items[it];
    // the model's trajectory count (a split model's chunks share it) and
    // this item's first trajectory in it
    const int64_t U = item.model_n_traj > 0 ? item.model_n_traj : item.n_traj;
    const int64_t cb = item.model_n_traj > 0 ? item.chunk_begin : 0;
    const uint32_t* blob = gblobs + item.blob_offset;
    const int words = (int)__ldg(blob + PYST_H_WORDS);
    const bool ok = stage_blob(sblob, blob, words, bar, parity,
                               ra.stage_polls);
    if (!ok) {
      mbar_drain(bar, parity);
      for (int64_t v = threadIdx.x; v < item.n_traj; v += bs)
        mark_staging_failure(ob, item.traj_offset + cb + v);
      break;
    }
    parity ^= 1u;
    ModelView m;
    m.load(sblob);
    if (SCORE && ob.score && m.nlaw > 0) {
      // (block-uniform) scores need a_j proportional to rate_j (mass
      // action): the item is not simulated; its samples read -1 and its
      // scores NaN
      const int KF = m.kappa * m.ita;
      const double nan = __longlong_as_double(0x7ff8000000000000ll);
      for (int64_t v = threadIdx.x; v < item.n_traj; v += bs) {
        const TrajOut o = ob.at(item.sample_offset, cb + v, item.traj_offset,
                                item.score_offset, U, m.R);
        for (int kf = 0; kf < KF; ++kf) o.samples[(int64_t)kf * o.stride] = -1;
        if (o.status) *o.status = (uint8_t)PYST_TRAJ_UNSUPPORTED;
        if (o.events) *o.events = 0;
        if (o.seqhash) *o.seqhash = 0;
        if (o.t_final) *o.t_final = 0.0;
        for (int j = 0; j < m.R; ++j) o.score[j] = nan;
      }
    } else {
      if (item.mapping == PYST_MAP_THREAD &&
          packed_bytes(m.R) <= (size_t)pk_bytes) {
        // (uniform over the block: every thread reads the same item)
        m.pk = spk;
        m.fast = __syncthreads_and(pack_reactions(m, spk)) != 0;
      }
      const bool tau = item.method == PYST_METHOD_TAU_LEAP;
      if (item.mapping == PYST_MAP_THREAD) {
        int32_t* xcol = (int32_t*)dyn + threadIdx.x;
        int64_t* slot =
            (int64_t*)((int32_t*)dyn + (size_t)m.S * bs) + threadIdx.x;
        for (int64_t v = threadIdx.x; v < item.n_traj; v += bs) {
          const int64_t u = cb + v;
          const TrajOut o = ob.at(item.sample_offset, u, item.traj_offset,
                                  item.score_offset, U, m.R);
          const uint64_t id = (uint64_t)item.traj_id_base + (uint64_t)u;
          if (m.fast && m.R >= 2 && m.R <= 8) {
            // (block-uniform) a packable item of 2 to 8 reactions: the
            // reaction count fixed at compile time (the 16,384-set sweep's
            // Lotka-Volterra and Schlogl items: 2,048 sets 3.86 -> 2.86 s)
            switch (m.R) {
#define PYST_EXACT_CASE(r)                                                 \
  case r:                                                                  \
    if (tau)                                                               \
      run_thread<r, true, SCORE, kPkPacked, r>(m, xcol, slot, bs, ra, id, \
                                               o);                         \
    else                                                                   \
      run_thread<r, false, SCORE, kPkPacked, r>(m, xcol, slot, bs, ra, id, \
                                                o);                        \
    break;
              PYST_EXACT_CASE(2)
              PYST_EXACT_CASE(3)
              PYST_EXACT_CASE(4)
              PYST_EXACT_CASE(5)
              PYST_EXACT_CASE(6)
              PYST_EXACT_CASE(7)
              PYST_EXACT_CASE(8)
#undef PYST_EXACT_CASE
            }
          } else if (m.R <= 8) {
            if (tau) run_thread<8, true, SCORE>(m, xcol, slot, bs, ra, id, o);
            else run_thread<8, false, SCORE>(m, xcol, slot, bs, ra, id, o);
          } else if (SCORE || m.R <= PYST_THREAD_MAX_REACTIONS) {
            // (the host maps scored items with more reactions to warps)
            if (tau) run_thread<32, true, SCORE>(m, xcol, slot, bs, ra, id, o);
            else run_thread<32, false, SCORE>(m, xcol, slot, bs, ra, id, o);
          } else {
            if (tau) run_thread_big<true>(m, xcol, slot, bs, ra, id, o);
            else run_thread_big<false>(m, xcol, slot, bs, ra, id, o);
          }
        }
      } else {
        unsigned char* mine = dyn + (size_t)wid * warp_bytes;
        const WarpSmem ws = warp_smem(mine, m.S, m.R);
        double* sacc = (double*)(mine + warp_smem_bytes(m.S, m.R));
        for (int64_t v = wid; v < item.n_traj; v += nw) {
          const int64_t u = cb + v;
          const TrajOut o = ob.at(item.sample_offset, u, item.traj_offset,
                                  item.score_offset, U, m.R);
          const uint64_t id = (uint64_t)item.traj_id_base + (uint64_t)u;
          if (tau) run_warp<true, SCORE>(m, ws, ra, id, o, sacc);
          else run_warp<false, SCORE>(m, ws, ra, id, o, sacc);
        }
      }
    }
    if (ob.stats || ob.jac) {
      // a split model: every thread makes its outputs visible device-wide
      // before the chunk is counted (uniform branch)
      if (item.group_chunks > 1) __threadfence();
      __syncthreads();  // the item's samples are all written
      bool last = true;
      if (item.group_chunks > 1) {
        // the block finishing the model's last chunk reduces the model
        if (threadIdx.x == 0) {
          s_last = atomicAdd(done + item.group, 1u) + 1u ==
                   (unsigned)item.group_chunks;
          if (s_last) __threadfence();
        }
        __syncthreads();
        last = s_last != 0;
      }
      if (last) item_epilogue(m, item, U, ob, (double*)dyn, dyn_bytes);
    }
    __syncthreads();  // everyone done with sblob and dyn before restaging
  }
}

}  // namespace (flavour)
using namespace PYST_CAT(batch_flavour_, PYST_SCORE, );

int PYST_CAT(launch_batch_, PYST_SCORE, )(
    const uint32_t* d_blobs, const pyst_batch_item* d_items, int64_t n_items,
    const pyst_batch_limits* lim, const RunArgs& ra, const OutBase& ob,
    unsigned long long* queue, unsigned* done, int bs, cudaStream_t st) {
  const size_t wb =
      host_warp_bytes(lim->max_species, lim->max_reactions, PYST_SCORE);
  const size_t thread_bytes = (size_t)bs * lim->max_species * 12;
  const size_t wbytes = wb * (size_t)(bs / 32);
  const size_t dyn = thread_bytes > wbytes ? thread_bytes : wbytes;
  const int maxr_pk = lim->max_reactions < PYST_THREAD_MAX_REACTIONS
                          ? lim->max_reactions
                          : PYST_THREAD_MAX_REACTIONS;
  const size_t pk_bytes = packed_bytes(maxr_pk);
  const size_t smem = (size_t)lim->max_blob_words * 4 + 16 + pk_bytes + dyn;
  if (smem > kMaxDynSmem) return PYST_EUNSUPPORTED;
  auto kf = k_batch<(bool)PYST_SCORE>;
  const int rc = set_smem(kf, smem);
  if (rc) return rc;
  if (cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st) !=
      cudaSuccess)
    return PYST_ECUDA;
  int per_sm = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kf, bs, smem);
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)num_sms() * per_sm;
  if (grid > n_items) grid = n_items;
  kf<<<(unsigned)grid, bs, smem, st>>>(d_blobs, d_items, n_items, ra, ob,
                                       queue, done, lim->max_blob_words,
                                       (int)wb, (int)dyn, (int)pk_bytes);
  return cudaGetLastError() == cudaSuccess ? PYST_OK : PYST_ECUDA;
}

}  // namespace pyst
