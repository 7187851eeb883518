/*
 * pystoch_b200.h -- C ABI of the B200 stochastic-simulation engine.
 *
 * The engine replaces the simulator layer of py_stoch (reference paths
 * below are relative to the reference project).  Every entry point takes
 * plain pointers and sizes; device pointers must be CUDA device memory
 * owned by the caller, and `stream` is a cudaStream_t passed as void*.
 * The library allocates no device memory on any entry point: scratch is
 * caller-provided workspace whose size the *_workspace_size functions
 * return.  Calls are stream-ordered and return before the GPU finishes.
 *
 * Replaces:
 *   CuGillespie.run        mod/simulator/cuGillespie/cuGillespie.py:16-46
 *                          (kernel_Gillespie, gillespie.py:27-149)
 *   CuTauLeaping.run       mod/simulator/cuTauLeaping/cuTauLeaping.py:18-84
 *                          (kernel_P1_P2, P1_P2.py:54-297;
 *                           kernel_P3, P3.py:29-163;
 *                           termination sum, cuTauLeaping.py:72)
 *   init_rng               mod/simulator/simulator.py:62-96
 *                          (replaced by the stateless Philox4x32-10 stream)
 *   __constant__ uploads   cuTauLeaping.py:86-107, cuGillespie.py:49-63
 *                          (replaced by the model blob, pyst_model_build)
 *   calculate_sizes        simulator.py:11-58, cuTauLeaping.py:162-214
 *                          (launch geometry is chosen inside the library)
 */
#ifndef PYSTOCH_B200_H
#define PYSTOCH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PYST_ABI_VERSION 3

/* ---- return codes ------------------------------------------------------ */
enum {
  PYST_OK = 0,
  PYST_EINVAL = 1,        /* bad argument (null pointer, size, alignment)   */
  PYST_ECUDA = 2,         /* a CUDA runtime call failed                     */
  PYST_EUNSUPPORTED = 3,  /* model exceeds a kernel limit (see below)       */
  PYST_EWORKSPACE = 4,    /* workspace smaller than *_workspace_size        */
  PYST_ETRAJ = 5          /* some trajectory ended with an error status     */
};

/* ---- per-trajectory status (uint8 array written by the run calls) ----- */
enum {
  PYST_TRAJ_DONE = 0,         /* reached the last sample time              */
  PYST_TRAJ_ABSORBED = 1,     /* total propensity hit 0; samples filled    */
  PYST_TRAJ_STEP_BUDGET = 2,  /* step budget exhausted; rest filled -1     */
  PYST_TRAJ_OVERFLOW = 3,     /* a species count would leave int32 range   */
  PYST_TRAJ_LEAP_RETRY = 4,   /* tau halved max_leap_retries times         */
  PYST_TRAJ_SAMPLER = 5,      /* Poisson sampler hit its iteration limit   */
  PYST_TRAJ_STAGING = 6,      /* model staging into shared memory timed out */
  PYST_TRAJ_RATE = 7,         /* a kinetic law gave a negative, infinite or
                                 NaN propensity                            */
  PYST_TRAJ_UNSUPPORTED = 8   /* batched run with scores: the item's model
                                 has general kinetic laws, so it was not
                                 simulated (samples -1, scores NaN)        */
};

/* ---- methods and mappings ---------------------------------------------- */
enum { PYST_METHOD_DIRECT = 0, PYST_METHOD_TAU_LEAP = 1 };
enum { PYST_MAP_AUTO = 0, PYST_MAP_THREAD = 1, PYST_MAP_WARP = 2 };

/* pyst_run_desc.flags bits.  PYST_FLAG_UNSORTED: run thread-mapped
 * tau-leaping with the simple one-trajectory-per-thread loop instead of the
 * default mode-sorted block scheduler (same results, slower). */
enum { PYST_FLAG_UNSORTED = 1 };

/* Limits of this library. */
#define PYST_MAX_SPECIES 1024
#define PYST_MAX_REACTIONS 4096
#define PYST_THREAD_MAX_REACTIONS 32  /* register-array thread kernels; above
                                         it the thread mapping recomputes
                                         propensities (no scores) */
#define PYST_MAX_BLOB_WORDS 12288     /* model blob staged in 48 KiB smem   */

/*
 * Model description (host pointers).  Matrices are dense, row-major
 * [species][reaction], the layout of SPN.Pre / SPN.Post
 * (mod/petri_net/SPN.py:72-97).
 *
 * Propensity of reaction j, mass-action form:
 *   a_j(x) = rate[j] * prod_i prod_{m < order[i][j]} (x_i - m * falling[i][j])
 * computed in FP32 in species order, factors in m order.
 *
 * General kinetic laws (the reference pastes any hazard as C source,
 * mod/parser/parser.py:32-55): reaction j with law_ptr[j+1] > law_ptr[j]
 * evaluates the postfix program law_code[law_ptr[j] .. law_ptr[j+1]) in FP64
 * and rounds the result to FP32 (its order column and rate are unused).
 * Program words are op << 24 | arg:
 *   1 X i (push x_i)   2 C k (push law_const[k])   3 ADD  4 SUB  5 MUL
 *   6 DIV   7 IDIV (C integer division: truncate toward zero)   8 NEG
 *   10 EXP  11 LN  12 SQRT  13 ABS  14 FLOOR  15 CEIL  16 DUP
 * at most 8 values deep.  law_ptr == NULL: every reaction is mass action.
 */
typedef struct pyst_model_desc {
  int32_t n_species;           /* S = TlArgs.N                              */
  int32_t n_reactions;         /* R = TlArgs.M                              */
  const int32_t* order;        /* [S*R] propensity order per species        */
  const uint8_t* falling;      /* [S*R] 1 falling factorial, 0 power; NULL=1 */
  const int32_t* pre;          /* [S*R] SPN.Pre (reactant species set)      */
  const int32_t* net_change;   /* [S*R] SPN.Post - SPN.Pre (TlArgs.V dense) */
  const double* rate;          /* [R] effective rate constants              */
  const int32_t* x0;           /* [S] TlArgs.x_0                            */
  const int32_t* hor;          /* [S] TlArgs.H                              */
  const int32_t* hor_type;     /* [S] TlArgs.H_type                         */
  const float* sample_times;   /* [ita] TlArgs.I (float32, ascending)       */
  int32_t n_samples;           /* ita                                       */
  const int32_t* out_species;  /* [kappa] TlArgs.E                          */
  int32_t n_out;               /* kappa                                     */
  double t_max;                /* TlArgs.t_max                              */
  float eta;                   /* TlArgs.eta (0.03)                         */
  int32_t n_c;                 /* TlArgs.n_c (10)                           */
  const int32_t* law_ptr;      /* [R+1] program ranges, or NULL              */
  const uint32_t* law_code;    /* [law_ptr[R]] program words                 */
  const double* law_const;     /* [n_law_const]                              */
  int32_t n_law_const;
} pyst_model_desc;

/* Run description.  Trajectory u (0 <= u < n_traj) draws from the Philox
 * stream keyed by `seed` with counter words (block index, block index >> 32,
 * id, id >> 32) where id = traj_id_base + u. */
typedef struct pyst_run_desc {
  int64_t n_traj;              /* U                                         */
  int64_t traj_id_base;        /* global id of trajectory 0                 */
  uint64_t seed;               /* Philox key                                */
  int32_t method;              /* PYST_METHOD_*                             */
  int32_t mapping;             /* PYST_MAP_*                                */
  int32_t ssa_fallback_steps;  /* SSA steps per fallback round (100)        */
  int32_t max_leap_retries;    /* tau halvings before giving up (64)        */
  int64_t step_budget;         /* max steps per trajectory (0 = 2^62)       */
  int32_t block_size;          /* 0 = library default                       */
  int32_t flags;               /* PYST_FLAG_* bits                          */
  /* Geometry of the mode-sorted tau-leaping kernel (thread mapping); 0
   * takes the default.  Results do not depend on it, only the speed. */
  int32_t round_ssa;           /* SSA steps per scheduling round (32)       */
  int32_t round_leap;          /* leaps per scheduling round (3)            */
  int32_t pool_slots;          /* trajectory slots per thread: 1 or 2 (2)   */
  int32_t sorted_block;        /* threads per block: 64..896, a multiple of
                                  32 (896; smaller when the pools do not fit
                                  shared memory)                            */
} pyst_run_desc;

/* Outputs (device pointers).  `samples` is required, the rest optional. */
typedef struct pyst_outputs {
  int32_t* samples;   /* [kappa][ita][out_stride], trajectory innermost     */
  int64_t out_stride; /* >= n_traj; 0 means n_traj                          */
  uint8_t* status;    /* [n_traj] PYST_TRAJ_*                               */
  int64_t* events;    /* [n_traj] reaction firings                          */
  uint64_t* seqhash;  /* [n_traj] FNV-1a hash of the firing sequence        */
  double* t_final;    /* [n_traj] clock when the trajectory stopped         */
  double* score;      /* [n_traj][R] d log p / d log rate_j; mass-action
                         models only (the run calls return
                         PYST_EUNSUPPORTED for a model with general
                         kinetic laws, batched runs mark such an item's
                         trajectories PYST_TRAJ_UNSUPPORTED)               */
  double* stats;      /* batched runs: per item [kappa][ita][3] mean,
                         variance, lag-1 correlation with the next sample */
  double* jacobian;   /* batched runs with scores: per item [2][kappa][ita][R]
                         d mean / d log rate_j, d variance / d log rate_j  */
} pyst_outputs;

/* ---- model blob (host side, no CUDA) ----------------------------------- */

/* Number of 32-bit words of the packed model (a multiple of 4). */
int pyst_model_blob_words(const pyst_model_desc* model, int64_t* n_words);

/* Pack `model` into `blob` (host memory, n_words words).  The caller copies
 * the blob to 16-byte-aligned device memory for the run calls. */
int pyst_model_build(const pyst_model_desc* model, uint32_t* blob,
                     int64_t n_words);

/* ---- single-model runs -------------------------------------------------- */

/* Both single-model runs take the blob twice: `h_blob` (host copy; only
 * its header is read, to size the launch without a device round trip) and
 * `d_blob` (16-byte-aligned device copy the kernels stage).  `d_workspace`
 * (8-byte aligned, >= pyst_run_workspace_size bytes) holds the trajectory
 * work queue: launches size their grid to the GPU's resident capacity and a
 * thread (or warp) whose trajectory ends takes the next unstarted one.  A
 * workspace may be reused by consecutive calls on one stream, not by calls
 * that overlap. */
#define PYST_RUN_WORKSPACE_BYTES 256
int pyst_run_workspace_size(const pyst_run_desc* run, size_t* bytes);

/* Direct-method SSA (Gillespie), one trajectory per thread or per warp.
 * Replaces CuGillespie.run and the forced-SSA path of CuTauLeaping.run
 * (gillespie=1, P1_P2.py:68-74 + P3.py:71-151). */
int pyst_ssa_direct_run(const uint32_t* h_blob, const uint32_t* d_blob,
                        const pyst_run_desc* run, const pyst_outputs* out,
                        void* d_workspace, size_t workspace_bytes,
                        void* stream);

/* Adaptive tau-leaping with critical reactions and SSA fallback, all
 * rounds inside one launch.  Replaces CuTauLeaping.run (host round loop
 * cuTauLeaping.py:49-76 with kernel_P1_P2 and kernel_P3). */
int pyst_tau_leap_run(const uint32_t* h_blob, const uint32_t* d_blob,
                      const pyst_run_desc* run, const pyst_outputs* out,
                      void* d_workspace, size_t workspace_bytes,
                      void* stream);

/* ---- batched persistent runs -------------------------------------------- */

/* One work item: a model, its trajectories and where its outputs go.
 * Offsets are in elements of the corresponding output arrays; a model's
 * samples are [kappa][ita][U] starting at sample_offset, U its trajectory
 * count.  A model may be split into chunks (consecutive items with the
 * same offsets): chunk c runs the model's trajectories chunk_begin ..
 * chunk_begin + n_traj - 1 of U = model_n_traj, so several blocks share a
 * large model; the block that finishes the model's last chunk computes its
 * statistics.  An unsplit model has chunk_begin 0 and model_n_traj 0. */
typedef struct pyst_batch_item {
  int64_t blob_offset;     /* word offset of the model blob in d_blobs     */
  int64_t n_traj;          /* trajectories of this item                    */
  int64_t traj_id_base;    /* Philox id of the model's trajectory 0        */
  int64_t sample_offset;   /* element offset of the model's [kappa][ita][U]*/
  int64_t traj_offset;     /* element offset into status/events/... arrays */
  int64_t score_offset;    /* element offset into score ([U][R])           */
  int64_t stats_offset;    /* element offset into stats                    */
  int64_t jac_offset;      /* element offset into jacobian                 */
  int32_t method;          /* PYST_METHOD_*                                */
  int32_t mapping;         /* PYST_MAP_THREAD or PYST_MAP_WARP             */
  int64_t chunk_begin;     /* first trajectory of this chunk in its model  */
  int64_t model_n_traj;    /* U of a split model (0: unsplit, U = n_traj)  */
  int32_t group;           /* split model: its completion counter,
                              0 <= group < n_items, one per model           */
  int32_t group_chunks;    /* split model: its number of chunks (0 or 1:
                              unsplit)                                      */
} pyst_batch_item;

/* Largest model of a batch (sizes the shared-memory layout). */
typedef struct pyst_batch_limits {
  int32_t max_blob_words;
  int32_t max_species;
  int32_t max_reactions;
  int32_t reserved;
} pyst_batch_limits;

/* Workspace bytes pyst_batch_run needs for n_items items: the work-queue
 * counter and one completion counter per item (split models). */
int pyst_batch_workspace_size(int64_t n_items, size_t* bytes);

/* Run every item in one persistent launch.  `d_items` is device memory
 * holding n_items pyst_batch_item; blocks take items from a device work
 * queue in array order (put expensive items first).  Per-trajectory output
 * pointers in `out` are bases that the item offsets index.  The run fields
 * n_traj, traj_id_base, method and mapping are taken from the items.
 * When `out->stats` / `out->jacobian` are set, the block that ran an item
 * reduces its samples (and scores) into the item's summary statistics and
 * their likelihood-ratio Jacobians in the same launch, in a fixed order.
 * Variances are population variances; the lag-1 entry of sample f is the
 * correlation of samples f and f+1 across trajectories (0 for the last
 * sample or a zero variance). */
int pyst_batch_run(const uint32_t* d_blobs, const pyst_batch_item* d_items,
                   int64_t n_items, const pyst_batch_limits* limits,
                   const pyst_run_desc* run, const pyst_outputs* out,
                   void* d_workspace, size_t workspace_bytes, void* stream);

/* ---- likelihood-ratio gradient ------------------------------------------ */

/* grad[j] = (1/U) sum_u h_u * score[u][j] with
 *   h_u = sum_{k,f} gmean[k][f] (O[k][f][u] - mean[k][f])
 *                 + gvar[k][f] ((O[k][f][u] - mean[k][f])^2 - var[k][f]).
 * `samples` is [kappa][ita][U] int32, `score` [U][R] double; mean, var,
 * gmean, gvar are [kappa][ita] double (gvar may be NULL).  Writes R doubles
 * to d_grad.  Deterministic: fixed reduction order for a given U. */
int pyst_score_backward_workspace_size(int64_t n_traj, int32_t n_reactions,
                                       size_t* bytes);
int pyst_score_backward(const int32_t* samples, const double* score,
                        int64_t n_traj, int32_t kappa, int32_t ita,
                        int32_t n_reactions, const double* mean,
                        const double* var, const double* gmean,
                        const double* gvar, double* d_grad,
                        void* d_workspace, size_t workspace_bytes,
                        void* stream);

/* ---- sufficient statistics for trajectories split across GPUs --------- */

/* The reference's only cross-trajectory reduction is the termination sum
 * gpuarray.sum(d_Q) (mod/simulator/cuTauLeaping/cuTauLeaping.py:72).  These
 * four calls extend it to the sample moments and their likelihood-ratio
 * gradients, in a form that gives the same bits however the trajectories
 * are split across GPUs (each GPU running a contiguous range of global
 * Philox ids):
 *
 *   pyst_sample_sums        per GPU: exact integer sums over its
 *                           trajectories, summed across GPUs with an
 *                           integer all-reduce (order-free, exact);
 *   pyst_moments_from_sums  every GPU: mean and variance from the totals;
 *   pyst_score_partials     per GPU: the backward reduction's partial sums,
 *                           one row of R per PYST_SCORE_CHUNK trajectories;
 *   pyst_score_combine      every GPU, after gathering all rows in global
 *                           trajectory order: the gradient.
 *
 * With ranges that start on multiples of PYST_SCORE_CHUNK, the moments and
 * gradient equal those of one GPU running every trajectory (pyst_score_
 * backward = pyst_score_partials + pyst_score_combine), bit for bit. */
#define PYST_SCORE_CHUNK 256
#define PYST_SUMS_MAX_TRAJ 2147483647LL

/* d_sums[kf][3] (int64, kf < kappa*ita) = sum over u < n_traj of x, of
 * (x*x) >> 32 and of (x*x) & 0xFFFFFFFF, x = samples[kf*stride + u]
 * (stride 0: n_traj).  Exact for n_traj <= PYST_SUMS_MAX_TRAJ. */
int pyst_sample_sums(const int32_t* samples, int64_t n_traj, int64_t stride,
                     int32_t kappa, int32_t ita, int64_t* d_sums,
                     void* stream);

/* d_mean[kf] = sx / n_total, d_var[kf] = (hi * 2^32 + lo) / n_total -
 * mean^2 (population variance) from the n_rows rows of d_sums. */
int pyst_moments_from_sums(const int64_t* d_sums, int32_t n_rows,
                           int64_t n_total, double* d_mean, double* d_var,
                           void* stream);

/* d_part[b][j] = sum over trajectories u of chunk b (PYST_SCORE_CHUNK of
 * them, in order) of h_u * score[u][j], h_u as in pyst_score_backward;
 * ceil(n_traj / PYST_SCORE_CHUNK) rows of n_reactions doubles. */
int pyst_score_partials(const int32_t* samples, const double* score,
                        int64_t n_traj, int32_t kappa, int32_t ita,
                        int32_t n_reactions, const double* mean,
                        const double* var, const double* gmean,
                        const double* gvar, double* d_part, void* stream);

/* d_grad[j] = (sum over the n_blocks rows of d_part, in row order) /
 * n_total. */
int pyst_score_combine(const double* d_part, int64_t n_blocks,
                       int32_t n_reactions, int64_t n_total, double* d_grad,
                       void* stream);

/* Same reduction as pyst_score_backward, for callers that cannot allocate
 * the workspace themselves: a host runtime that has already handed all
 * device memory to its own pool, or a loop that cannot accept the
 * device-wide synchronisation a cudaMalloc may cause.  It allocates nothing
 * (no cudaMalloc, cudaFree or allocating library call); its scratch is a
 * fixed PYST_NOALLOC_SCRATCH_BYTES array inside the library that every GPU
 * loading the library keeps until exit.  Calls needing more scratch than
 * that -- ceil(n_traj / 256) * n_reactions * 8 bytes, i.e. n_traj up to
 * 1,048,576 with 32 reactions -- return PYST_EUNSUPPORTED.  The first call
 * on a device looks up the array's device address there (make that first
 * call before any stream capture) and keeps it for the life of the
 * process, which assumes the device's primary context lives as long: after
 * a cudaDeviceReset, reload the library.  All calls share the one array, which
 * keeps the last call's contents; calls that overlap on the GPU race, so
 * serialise them (one stream, or events).  This entry point has no
 * counterpart in the reference, which has no gradients. */
#define PYST_NOALLOC_SCRATCH_BYTES (1 << 20)
int pyst_score_backward_noalloc(const int32_t* samples, const double* score,
                                int64_t n_traj, int32_t kappa, int32_t ita,
                                int32_t n_reactions, const double* mean,
                                const double* var, const double* gmean,
                                const double* gvar, double* d_grad,
                                void* stream);

/* ---- misc -------------------------------------------------------------- */

int pyst_abi_version(void);
const char* pyst_status_string(int code);
const char* pyst_traj_status_string(int code);

/* Blob header layout (word indices), shared by the packer and kernels. */
enum {
  PYST_H_MAGIC = 0,      /* 0x31545950 */
  PYST_H_WORDS = 1,
  PYST_H_S = 2,
  PYST_H_R = 3,
  PYST_H_KAPPA = 4,
  PYST_H_ITA = 5,
  PYST_H_NFAC = 6,
  PYST_H_NNET = 7,
  PYST_H_NSPV = 8,
  PYST_H_NCRIT = 9,
  PYST_H_OFF_RATE = 10,     /* f32[R]                                       */
  PYST_H_OFF_FACPTR = 11,   /* i32[R+1]                                     */
  PYST_H_OFF_FAC = 12,      /* species | order<<16 | falling<<24            */
  PYST_H_OFF_NETPTR = 13,   /* i32[R+1]                                     */
  PYST_H_OFF_NET = 14,      /* species | (int16 delta)<<16                  */
  PYST_H_OFF_TIMES = 15,    /* f32[ita]                                     */
  PYST_H_OFF_OUT = 16,      /* i32[kappa]                                   */
  PYST_H_OFF_X0 = 17,       /* i32[S]                                       */
  PYST_H_OFF_SPVPTR = 18,   /* i32[S+1] species-major V of reactant species */
  PYST_H_OFF_SPV = 19,      /* reaction | (int16 v)<<16                     */
  PYST_H_OFF_G = 20,        /* H | H_type<<8 | reactant<<16                 */
  PYST_H_OFF_CRITPTR = 21,  /* i32[R+1]                                     */
  PYST_H_OFF_CRIT = 22,     /* species | |v|<<16 (entries with v < 0)       */
  PYST_H_NC = 23,
  PYST_H_ETA = 24,          /* f32 bits                                     */
  PYST_H_FLAGS = 25,
  PYST_H_TMAX_LO = 26,      /* f64 bits                                     */
  PYST_H_TMAX_HI = 27,
  PYST_H_OFF_LAWPTR = 28,   /* i32[R+1] kinetic-law program ranges          */
  PYST_H_OFF_LAW = 29,      /* program words                                */
  PYST_H_OFF_LAWC = 30,     /* f64[] constants (even word offset)           */
  PYST_H_NLAW = 31,         /* reactions with a program (0: none)           */
  PYST_H_WORDS_HEADER = 32
};
#define PYST_BLOB_MAGIC 0x31545950u

#ifdef __cplusplus
}
#endif
#endif
