/*
 * pystoch_b200_testing.h -- test hooks exported by libpystoch_b200.so.
 *
 * Not part of the drop-in surface: they expose the device random-number
 * generator and elementary functions so tests can compare them bit for bit
 * with the host oracle and with published known-answer vectors.
 */
#ifndef PYSTOCH_B200_TESTING_H
#define PYSTOCH_B200_TESTING_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* count Philox blocks of the stream (seed, id) from block index n0;
 * d_out holds 4*count words. */
int pyst_test_philox(uint64_t seed, uint64_t id, uint64_t n0, int64_t count,
                     uint32_t* d_out, void* stream);

/* Philox4x32-10 of raw (counter[4], key[2]) rows, 6 words each; with
 * use_curand != 0 the CUDA toolkit's curand_Philox4x32_10 computes them. */
int pyst_test_philox_raw(const uint32_t* d_ctr_key, int64_t count,
                         uint32_t* d_out, int use_curand, void* stream);

/* which: 0 pyst_log, 1 pyst_exp, 2 log-factorial, 3 CUDA log, 4 CUDA exp. */
int pyst_test_math(const double* d_x, int64_t n, int which, double* d_out,
                   void* stream);

/* Poisson draw i with lambda d_lam[i], trajectory id i, leap index 7,
 * reaction i mod 1024, retry 3. */
int pyst_test_poisson(const float* d_lam, int64_t n, uint64_t seed,
                      int32_t* d_out, void* stream);

/* Issue-rate probe of one arithmetic pipe (the denominators of the
 * instruction roofline): `blocks` blocks of 256 threads each run `iters`
 * iterations of 8 independent chains of one operation -- which 0 FP32
 * fma, 1 INT32 multiply-add, 2 FP64 fma, 3 INT32 xor + add (two ALU
 * operations) -- and write one double per thread to d_sink.  The caller
 * times it: 8 * iters * 256 * blocks chain steps. */
int pyst_test_pipe(int32_t which, int32_t iters, int32_t blocks,
                   double* d_sink, void* stream);

/* 1 if every reaction of the host blob fits the packed per-reaction
 * descriptors (the host's choice of the lane-tree kernel), 0 if not,
 * minus a PYST_E* code for a bad blob. */
int pyst_test_model_packable(const uint32_t* h_blob);

/* Bound of the model-staging wait of every later run call in this process
 * (polls of the staging mbarrier; PYST_MBAR_POLL_LIMIT by default).  With
 * 0 every staging wait gives up at once, so a test can see the timeout
 * path run: each block then waits, bounded, for its in-flight copy before
 * moving on, and marks its trajectories PYST_TRAJ_STAGING.  polls < 0
 * restores the default.  Returns the previous bound. */
int pyst_test_set_staging_polls(int32_t polls);

#ifdef __cplusplus
}
#endif
#endif
