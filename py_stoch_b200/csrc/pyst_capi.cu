// C ABI of libpystoch_b200.so (include/pystoch_b200.h): argument checks,
// launch-geometry choice and dispatch to the kernel translation units.
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "pyst_launch.cuh"
#include "pystoch_b200.h"
#include "pystoch_b200_testing.h"

namespace pyst {

int num_sms() {
  static std::atomic<int> cached{0};
  int n = cached.load();
  if (n) return n;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
          cudaSuccess ||
      n <= 0)
    return 148;
  cached.store(n);
  return n;
}

}  // namespace pyst

using namespace pyst;

namespace {

// Round lengths of the mode-sorted tau-leaping kernel: SSA steps and leaps
// a trajectory advances between two regroupings of its block.  On the
// Schlogl workload (262144 trajectories, 896-thread blocks, SSA fallback
// rounds of 100 steps) 40 / 4 measured 64.3 ms a step, 20 / 2 64.5,
// 50 / 5 64.6, 40 / 3 65.7, 60 / 6 66.1, 30 / 3 66.6, 32 / 3 68.3, 36 / 4
// 69.2, 48 / 4 69.1, 45 / 4 70.0, 10 / 1 71.1 (a comb in the SSA length:
// where the fallback's 100th step, and with it the DECIDE that may switch
// the trajectory out of its SSA warp, falls within a round sets how long
// lanes idle); with 1024-thread blocks longer rounds were slower still
// (128 / 8 100, 256 / 16 107, 256 / 32 121, earlier kernels), and resizing
// leap rounds to match the SSA rounds' measured time was slower too.
#ifndef PYST_CAP_SSA
#define PYST_CAP_SSA 40
#endif
#ifndef PYST_CAP_LEAP
#define PYST_CAP_LEAP 4
#endif
constexpr int kSortedCapSsa = PYST_CAP_SSA;
// Auto mapping of networks with more reactions than the register engine:
// warps when the run has at most this many trajectories per SM.
constexpr int kWarpAutoPerSm = 32;
constexpr int kSortedCapLeap = PYST_CAP_LEAP;

// The factor and net-change sections of a host blob lie inside it (so the
// packability check below reads only the blob).
bool sections_in_blob(const uint32_t* h, int words, int R) {
  const int64_t fp = h[PYST_H_OFF_FACPTR], f = h[PYST_H_OFF_FAC];
  const int64_t np = h[PYST_H_OFF_NETPTR], n = h[PYST_H_OFF_NET];
  if (fp < PYST_H_WORDS_HEADER || fp + R + 1 > words ||
      np < PYST_H_WORDS_HEADER || np + R + 1 > words)
    return false;
  if (f < PYST_H_WORDS_HEADER || n < PYST_H_WORDS_HEADER) return false;
  for (int j = 0; j <= R; ++j)
    if (h[fp + j] > h[fp + R] || f + h[fp + j] > words ||
        h[np + j] > h[np + R] || n + h[np + j] > words)
      return false;
  return true;
}

int read_header(const uint32_t* h, HostModelInfo* mi) {
  if (!h) return PYST_EINVAL;
  if (h[PYST_H_MAGIC] != PYST_BLOB_MAGIC) return PYST_EINVAL;
  mi->words = (int)h[PYST_H_WORDS];
  mi->S = (int)h[PYST_H_S];
  mi->R = (int)h[PYST_H_R];
  mi->nlaw = (int)h[PYST_H_NLAW];
  if (mi->words <= 0 || (mi->words & 3) || mi->words > PYST_MAX_BLOB_WORDS)
    return PYST_EUNSUPPORTED;
  if (mi->S < 1 || mi->R < 1 || mi->S > PYST_MAX_SPECIES ||
      mi->R > PYST_MAX_REACTIONS)
    return PYST_EUNSUPPORTED;
  mi->packable = mi->nlaw == 0 && sections_in_blob(h, mi->words, mi->R);
  for (int j = 0; j < mi->R && mi->packable; ++j)
    mi->packable = blob_reaction_packable(h, j);
  return PYST_OK;
}

int check_run(const pyst_run_desc* run) {
  if (!run) return PYST_EINVAL;
  if (run->n_traj < 0 || run->traj_id_base < 0) return PYST_EINVAL;
  if (run->method != PYST_METHOD_DIRECT && run->method != PYST_METHOD_TAU_LEAP)
    return PYST_EINVAL;
  if (run->mapping < PYST_MAP_AUTO || run->mapping > PYST_MAP_WARP)
    return PYST_EINVAL;
  if (run->method == PYST_METHOD_TAU_LEAP &&
      (run->ssa_fallback_steps < 1 || run->max_leap_retries < 0 ||
       run->max_leap_retries > 63))
    return PYST_EINVAL;
  if (run->step_budget < 0) return PYST_EINVAL;
  if (run->block_size != 0 &&
      (run->block_size < 32 || run->block_size > 128 || run->block_size % 32))
    return PYST_EINVAL;
  if (run->round_ssa < 0 || run->round_leap < 0 || run->pool_slots < 0 ||
      run->pool_slots > 2 || run->sorted_block < 0 ||
      (run->sorted_block != 0 &&
       (run->sorted_block < 64 || run->sorted_block > 896 ||
        run->sorted_block % 32)))
    return PYST_EINVAL;
  return PYST_OK;
}

// Bound of the model-staging wait (pyst_test_set_staging_polls).
std::atomic<int> g_stage_polls{PYST_MBAR_POLL_LIMIT};

RunArgs make_args(const pyst_run_desc* run) {
  RunArgs ra;
  ra.stage_polls = g_stage_polls.load();
  ra.seed = run->seed;
  ra.step_budget = run->step_budget ? run->step_budget : (1ll << 62);
  ra.ssa_fallback_steps =
      run->ssa_fallback_steps > 0 ? run->ssa_fallback_steps : 100;
  ra.max_leap_retries = run->max_leap_retries;
  return ra;
}

OutBase make_outbase(const pyst_outputs* out, int64_t n_traj) {
  OutBase ob;
  ob.samples = out->samples;
  ob.stride = out->out_stride ? out->out_stride : n_traj;
  ob.status = out->status;
  ob.events = out->events;
  ob.seqhash = out->seqhash;
  ob.t_final = out->t_final;
  ob.score = out->score;
  ob.stats = out->stats;
  ob.jac = out->jacobian;
  return ob;
}

int single_run(const uint32_t* h_blob, const uint32_t* d_blob,
               const pyst_run_desc* run, const pyst_outputs* out,
               void* d_workspace, size_t workspace_bytes, void* stream,
               int method) {
  HostModelInfo mi;
  int rc = read_header(h_blob, &mi);
  if (rc) return rc;
  rc = check_run(run);
  if (rc) return rc;
  if (run->method != method) return PYST_EINVAL;
  if (!d_blob || ((uintptr_t)d_blob & 15)) return PYST_EINVAL;
  if (!out || !out->samples) return PYST_EINVAL;
  if (out->out_stride != 0 && out->out_stride < run->n_traj)
    return PYST_EINVAL;
  if (!d_workspace || ((uintptr_t)d_workspace & 7)) return PYST_EINVAL;
  if (workspace_bytes < PYST_RUN_WORKSPACE_BYTES) return PYST_EWORKSPACE;
  if (out->stats || out->jacobian) return PYST_EINVAL;  // batched runs only
  // a likelihood-ratio score N_j - int a_j dt is d log p / d log rate_j only
  // when a_j is proportional to rate_j (mass action); a general kinetic law
  // leaves the rate column unused
  if (out->score && mi.nlaw > 0) return PYST_EUNSUPPORTED;
  if (run->n_traj == 0) return PYST_OK;
  const RunArgs ra = make_args(run);
  const OutBase ob = make_outbase(out, run->n_traj);
  unsigned long long* queue = (unsigned long long*)d_workspace;
  cudaStream_t st = (cudaStream_t)stream;
  const bool tau = method == PYST_METHOD_TAU_LEAP;
  const bool score = out->score != nullptr;
  int mapping = run->mapping;
  const int bs = run->block_size ? run->block_size : 128;
  // auto: a thread per trajectory unless the species columns are large,
  // the scores' register accumulators do not fit, or a run of a large
  // network is too small to fill the GPU (a warp then spreads each step's
  // reactions over 32 lanes instead of looping over them in one thread)
  if (mapping == PYST_MAP_AUTO)
    mapping = (mi.S <= 64 && (mi.R <= PYST_THREAD_MAX_REACTIONS ||
                              (!score && run->n_traj > (int64_t)num_sms() *
                                                           kWarpAutoPerSm)))
                  ? PYST_MAP_THREAD
                  : PYST_MAP_WARP;
  // thread-mapped scores keep per-reaction accumulators in registers
  if (mapping == PYST_MAP_THREAD && score &&
      mi.R > PYST_THREAD_MAX_REACTIONS)
    return PYST_EUNSUPPORTED;
  const uint64_t idb = (uint64_t)run->traj_id_base;
  const int64_t n = run->n_traj;
  if (mapping == PYST_MAP_THREAD && tau &&
      !(run->flags & PYST_FLAG_UNSORTED) && mi.nlaw == 0) {
    // (models with general kinetic laws take the simple tau loop: the
    // sorted kernel's engine carries no law evaluator)
    SortedGeometry g;
    g.cap_ssa = run->round_ssa ? run->round_ssa : kSortedCapSsa;
    g.cap_leap = run->round_leap ? run->round_leap : kSortedCapLeap;
    g.pool = run->pool_slots;
    g.block = run->sorted_block;
    const int rc =
        score ? launch_tau_sorted_1(mi.R, d_blob, mi, n, idb, ra, ob, queue,
                                    g, st)
              : launch_tau_sorted_0(mi.R, d_blob, mi, n, idb, ra, ob, queue,
                                    g, st);
    // the sorted block keeps every slot's species in shared memory; for
    // models with too many species fall back to the unsorted loop
    if (rc != PYST_EUNSUPPORTED) return rc;
  }
  if (mapping == PYST_MAP_THREAD) {
    if (tau)
      return score ? launch_plain_thread_11(mi.R, d_blob, mi, n, idb, ra, ob,
                                            bs, queue, st)
                   : launch_plain_thread_10(mi.R, d_blob, mi, n, idb, ra, ob,
                                            bs, queue, st);
    return score ? launch_plain_thread_01(mi.R, d_blob, mi, n, idb, ra, ob, bs,
                                          queue, st)
                 : launch_plain_thread_00(mi.R, d_blob, mi, n, idb, ra, ob, bs,
                                          queue, st);
  }
  if (tau)
    return score ? launch_plain_warp_11(d_blob, mi, n, idb, ra, ob, bs, queue,
                                        st)
                 : launch_plain_warp_10(d_blob, mi, n, idb, ra, ob, bs, queue,
                                        st);
  return score ? launch_plain_warp_01(d_blob, mi, n, idb, ra, ob, bs, queue,
                                      st)
               : launch_plain_warp_00(d_blob, mi, n, idb, ra, ob, bs, queue,
                                      st);
}

}  // namespace

extern "C" {

int pyst_abi_version(void) { return PYST_ABI_VERSION; }

int pyst_test_model_packable(const uint32_t* h_blob) {
  HostModelInfo mi;
  const int rc = read_header(h_blob, &mi);
  if (rc) return -rc;
  return mi.packable ? 1 : 0;
}

int pyst_test_set_staging_polls(int32_t polls) {
  return g_stage_polls.exchange(polls < 0 ? PYST_MBAR_POLL_LIMIT : polls);
}

const char* pyst_status_string(int code) {
  switch (code) {
    case PYST_OK: return "ok";
    case PYST_EINVAL: return "invalid argument";
    case PYST_ECUDA: return "CUDA runtime error";
    case PYST_EUNSUPPORTED: return "model exceeds a kernel limit";
    case PYST_EWORKSPACE: return "workspace too small";
    case PYST_ETRAJ: return "a trajectory ended with an error status";
  }
  return "unknown status";
}

const char* pyst_traj_status_string(int code) {
  switch (code) {
    case PYST_TRAJ_DONE: return "done";
    case PYST_TRAJ_ABSORBED: return "absorbed (total propensity 0)";
    case PYST_TRAJ_STEP_BUDGET: return "step budget exhausted";
    case PYST_TRAJ_OVERFLOW: return "species count out of int32 range";
    case PYST_TRAJ_LEAP_RETRY: return "tau halved too many times";
    case PYST_TRAJ_SAMPLER: return "Poisson sampler iteration limit";
    case PYST_TRAJ_STAGING: return "model staging timed out";
    case PYST_TRAJ_RATE: return "kinetic law gave an invalid propensity";
    case PYST_TRAJ_UNSUPPORTED:
      return "scores requested for a model with general kinetic laws";
  }
  return "unknown trajectory status";
}

int pyst_run_workspace_size(const pyst_run_desc* run, size_t* bytes) {
  if (!run || !bytes) return PYST_EINVAL;
  *bytes = PYST_RUN_WORKSPACE_BYTES;
  return PYST_OK;
}

int pyst_ssa_direct_run(const uint32_t* h_blob, const uint32_t* d_blob,
                        const pyst_run_desc* run, const pyst_outputs* out,
                        void* d_workspace, size_t workspace_bytes,
                        void* stream) {
  return single_run(h_blob, d_blob, run, out, d_workspace, workspace_bytes,
                    stream, PYST_METHOD_DIRECT);
}

int pyst_tau_leap_run(const uint32_t* h_blob, const uint32_t* d_blob,
                      const pyst_run_desc* run, const pyst_outputs* out,
                      void* d_workspace, size_t workspace_bytes,
                      void* stream) {
  return single_run(h_blob, d_blob, run, out, d_workspace, workspace_bytes,
                    stream, PYST_METHOD_TAU_LEAP);
}

int pyst_batch_workspace_size(int64_t n_items, size_t* bytes) {
  if (!bytes || n_items < 0) return PYST_EINVAL;
  // the work-queue counter (padded), then one completion counter per item
  *bytes = PYST_RUN_WORKSPACE_BYTES + (size_t)n_items * sizeof(uint32_t);
  return PYST_OK;
}

int pyst_batch_run(const uint32_t* d_blobs, const pyst_batch_item* d_items,
                   int64_t n_items, const pyst_batch_limits* lim,
                   const pyst_run_desc* run, const pyst_outputs* out,
                   void* d_workspace, size_t workspace_bytes, void* stream) {
  if (!d_blobs || !d_items || !lim || !run || !out || !out->samples)
    return PYST_EINVAL;
  if (((uintptr_t)d_blobs & 15) || n_items < 0) return PYST_EINVAL;
  if (!d_workspace || ((uintptr_t)d_workspace & 7)) return PYST_EINVAL;
  if (workspace_bytes <
      PYST_RUN_WORKSPACE_BYTES + (size_t)n_items * sizeof(uint32_t))
    return PYST_EWORKSPACE;
  if (lim->max_blob_words <= 0 || (lim->max_blob_words & 3) ||
      lim->max_blob_words > PYST_MAX_BLOB_WORDS || lim->max_species < 1 ||
      lim->max_reactions < 1 || lim->max_species > PYST_MAX_SPECIES ||
      lim->max_reactions > PYST_MAX_REACTIONS)
    return PYST_EUNSUPPORTED;
  if (run->step_budget < 0 || run->ssa_fallback_steps < 1 ||
      run->max_leap_retries < 0 || run->max_leap_retries > 63)
    return PYST_EINVAL;
  if (out->jacobian && !out->score) return PYST_EINVAL;
  if (n_items == 0) return PYST_OK;
  const int bs = run->block_size ? run->block_size : 128;
  if (bs < 32 || bs > 128 || bs % 32) return PYST_EINVAL;
  const RunArgs ra = make_args(run);
  OutBase ob = make_outbase(out, 1);
  ob.stride = 0;  // per item
  cudaStream_t st = (cudaStream_t)stream;
  unsigned long long* queue = (unsigned long long*)d_workspace;
  unsigned* done =
      (unsigned*)((unsigned char*)d_workspace + PYST_RUN_WORKSPACE_BYTES);
  if (cudaMemsetAsync(done, 0, (size_t)n_items * sizeof(uint32_t), st) !=
      cudaSuccess)
    return PYST_ECUDA;
  if (out->score)
    return launch_batch_1(d_blobs, d_items, n_items, lim, ra, ob, queue, done,
                          bs, st);
  return launch_batch_0(d_blobs, d_items, n_items, lim, ra, ob, queue, done,
                        bs, st);
}

int pyst_score_backward_workspace_size(int64_t n_traj, int32_t n_reactions,
                                       size_t* bytes) {
  if (!bytes || n_traj < 0 || n_reactions < 1) return PYST_EINVAL;
  int64_t nblk = score_backward_blocks(n_traj);
  if (nblk < 1) nblk = 1;
  *bytes = (size_t)nblk * (size_t)n_reactions * sizeof(double);
  return PYST_OK;
}

int pyst_score_backward(const int32_t* samples, const double* score,
                        int64_t n_traj, int32_t kappa, int32_t ita,
                        int32_t n_reactions, const double* mean,
                        const double* var, const double* gmean,
                        const double* gvar, double* d_grad, void* d_workspace,
                        size_t workspace_bytes, void* stream) {
  if (!samples || !score || !mean || !gmean || !d_grad || n_traj < 1 ||
      kappa < 1 || ita < 1 || n_reactions < 1)
    return PYST_EINVAL;
  if (gvar && !var) return PYST_EINVAL;
  size_t need = 0;
  pyst_score_backward_workspace_size(n_traj, n_reactions, &need);
  if (!d_workspace || ((uintptr_t)d_workspace & 7)) return PYST_EINVAL;
  if (workspace_bytes < need) return PYST_EWORKSPACE;
  return launch_score_backward(samples, score, n_traj, kappa, ita,
                               n_reactions, mean, var, gmean, gvar,
                               (double*)d_workspace, d_grad,
                               (cudaStream_t)stream);
}

int pyst_sample_sums(const int32_t* samples, int64_t n_traj, int64_t stride,
                     int32_t kappa, int32_t ita, int64_t* d_sums,
                     void* stream) {
  if (!samples || !d_sums || n_traj < 0 || n_traj > PYST_SUMS_MAX_TRAJ ||
      kappa < 1 || ita < 1)
    return PYST_EINVAL;
  if (stride == 0) stride = n_traj;
  if (stride < n_traj) return PYST_EINVAL;
  return launch_sample_sums(samples, n_traj, stride, kappa * ita, d_sums,
                            (cudaStream_t)stream);
}

int pyst_moments_from_sums(const int64_t* d_sums, int32_t n_rows,
                           int64_t n_total, double* d_mean, double* d_var,
                           void* stream) {
  if (!d_sums || !d_mean || !d_var || n_rows < 1 || n_total < 1)
    return PYST_EINVAL;
  return launch_moments_from_sums(d_sums, n_rows, n_total, d_mean, d_var,
                                  (cudaStream_t)stream);
}

int pyst_score_partials(const int32_t* samples, const double* score,
                        int64_t n_traj, int32_t kappa, int32_t ita,
                        int32_t n_reactions, const double* mean,
                        const double* var, const double* gmean,
                        const double* gvar, double* d_part, void* stream) {
  if (!samples || !score || !mean || !gmean || !d_part || n_traj < 1 ||
      kappa < 1 || ita < 1 || n_reactions < 1)
    return PYST_EINVAL;
  if (gvar && !var) return PYST_EINVAL;
  return launch_score_partials(samples, score, n_traj, kappa, ita,
                               n_reactions, mean, var, gmean, gvar, d_part,
                               (cudaStream_t)stream);
}

int pyst_score_combine(const double* d_part, int64_t n_blocks,
                       int32_t n_reactions, int64_t n_total, double* d_grad,
                       void* stream) {
  if (!d_part || !d_grad || n_blocks < 1 || n_reactions < 1 || n_total < 1)
    return PYST_EINVAL;
  return launch_score_combine(d_part, n_blocks, n_reactions, n_total, d_grad,
                              (cudaStream_t)stream);
}

}  // extern "C"
