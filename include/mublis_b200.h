/*
 * mublis_b200.h -- B200-specific extensions of libmublis.
 *
 * None of these has a counterpart in the reference (a CPU library with no
 * device, streams or precision forms); they sit beside the unchanged
 * cblas.h / mublis.h entry points.  All return 0 on success, nonzero on
 * failure (1 invalid argument, 2 CUDA failure, 3 out of memory / refused,
 * 4 a bounded device wait gave up); mublis_b200_last_error() describes the
 * calling thread's last failure.
 */
#ifndef MUBLIS_B200_H
#define MUBLIS_B200_H

#include <stddef.h>
#include <stdint.h>

#include "mublis.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Brings up the device (also done lazily by the first call).  Fails when no
 * sm_100 device is present: the library has no CPU fallback. */
int mublis_b200_init(void);
const char *mublis_b200_last_error(void);

/* Per-thread stream.  Each host thread gets its own non-blocking stream by
 * default; set_stream makes the library issue the calling thread's work on
 * the given cudaStream_t instead (the caller keeps ownership).  Calls remain
 * synchronous: they return after their work on that stream completes. */
int mublis_b200_set_stream(void *cuda_stream);
void *mublis_b200_get_stream(void);

/* Precision form used by the routines of one precision ('s' or 'd'):
 *   's': "plain" (FP32 FMA pipe), "bf16x3" (tcgen05, hi/lo split, 3
 *        products, FP32 accumulate), "bf16x6" (3-term split, 6 products),
 *        "fp16x3" (per-row/column scaled fp16 hi/lo split, 3 products)
 *   'd': "plain" (FP64 tensor pipe, mma.sync .f64), "ozaki" or
 *        "ozaki:<slices>" (int8 slices, exact int32 tensor-core
 *        accumulation, FP64 recombination)
 *   both: "ozaki2" or "ozaki2:<moduli>" (int8 residues modulo up to 16
 *        moduli, exact int32 products, Chinese-remainder reconstruction;
 *        default 16 moduli for FP64, 8 for FP32)
 *   both: "ozaki2@<target>" (e.g. "ozaki2@1e-16") -- the modular form with
 *        the fewest moduli whose normwise error, measured on a calibration
 *        block of the call (mublis_b200_ozaki2_autotune), is within the
 *        target; the choice is cached per precision, power-of-two bucket of
 *        k and target (and saved in the tuned table)
 *   both: "auto" -- per call, the fastest form whose error is no worse than
 *        plain: FP32 uses fp16x3 when min(m, n) >= 4096 and k >= 2048,
 *        bf16x6 when min(m, n) and k are >= 512, FP64 uses
 *        ozaki2 when min(m, n) and k are >= 1024 and m * n >= 2048^2,
 *        plain otherwise
 * Also settable with MUBLIS_B200_SFORM / MUBLIS_B200_DFORM. */
int mublis_b200_set_form(char dtype, const char *form);

/* Launch accounting and per-kernel device timing.  profile_read writes
 * {"kernel": [launches, total_ms], ...} for launches since the last read. */
unsigned long long mublis_b200_launch_count(void);
int mublis_b200_profile_enable(int on);
int mublis_b200_profile_read(char *buf, unsigned long len);

/* Modulus-count autotuner of the modular Ozaki form.  For C = op(A) op(B)
 * (device pointers; m x n x k; strides as in mublis_{s,d}gemm), computes a
 * calibration block -- the leading min(m, 256) x min(n, 256) of the product
 * over the whole k -- with a compensated (Dot2) dot product on the device,
 * runs the form on it with 6 .. 16 moduli (FP32: 6 .. 8) from the fewest up
 * and picks the first whose normwise error ||C_N - C_ref||_F /
 * (||A_blk||_F ||B_blk||_F) is <= target_err (16 / 8 if none is).  The
 * choice is recorded for later "ozaki2@<target_err>" calls of the same
 * precision and power-of-two bucket of k.  *moduli gets the count,
 * *measured_err (may be NULL) its measured error.  dtype 's' or 'd'. */
int mublis_b200_ozaki2_autotune(char dtype, mublis_trans_t trans_a, mublis_trans_t trans_b, int m,
                                int n, int k, const void *a, int rs_a, int cs_a, const void *b,
                                int rs_b, int cs_b, double target_err, int *moduli,
                                double *measured_err);

/* Failure-detection test of the bounded device waits.  Arms a one-shot
 * stall for the next launch of the FP64 tensor-pipe GEMM kernel in the
 * process: that launch bounds its mbarrier waits by wait_limit_ns (at most
 * 2 s) instead of 2 s, and its producer issues no loads, so the consumers'
 * first wait runs out; the kernel raises its abort flag and error word and
 * returns (nothing faults, nothing spins unbounded), and the call that made
 * the launch returns 4.  Later launches run normally. */
int mublis_b200_test_stall_next(unsigned long long wait_limit_ns);

/* Seeded device fills (Philox4x32-10, key = (seed, matrix_id), counter =
 * column-major element index i + j*m; kind 0 uniform[-1,1), 1 wide
 * +-[1,2)*2^[-10,10], 2 uniform[1,2)).  x is a device pointer to an m x n
 * column-major matrix with leading dimension ld. */
int mublis_b200_fill_s(float *x, long m, long n, long ld, uint32_t seed, uint32_t matrix_id,
                       int kind);
int mublis_b200_fill_d(double *x, long m, long n, long ld, uint32_t seed, uint32_t matrix_id,
                       int kind);

/* ---- grouped launches (no counterpart in the reference, which runs one
 * call per host thread) -------------------------------------------------
 * Many independent problems of one precision ('s' or 'd') in one persistent
 * launch that walks a device-side problem table.  Operands must be device
 * pointers; column-major with leading dimensions; alpha/beta are taken at
 * the problem's precision.  Synchronous. */
typedef struct {
  int trans_a, trans_b; /* mublis_trans_t */
  int m, n, k;
  double alpha, beta;
  const void *a;
  int lda;
  const void *b;
  int ldb;
  void *c;
  int ldc;
} mublis_b200_gemm_problem_t;

/* Left-side solve op(A) X = alpha B, B overwritten (m x n, ldb). */
typedef struct {
  int uplo, trans_a, diag; /* mublis_uplo_t (LOWER/UPPER), mublis_trans_t, mublis_diag_t */
  int m, n;
  double alpha;
  const void *a;
  int lda;
  void *b;
  int ldb;
} mublis_b200_trsm_problem_t;

int mublis_b200_gemm_grouped(char dtype, const mublis_b200_gemm_problem_t *problems, int count);
int mublis_b200_trsm_grouped(char dtype, const mublis_b200_trsm_problem_t *problems, int count);

/* Plans: a grouped call over a fixed problem table (the same pointers and
 * sizes every run).  Creation autotunes the tile shape per size class by
 * timing every variant on the actual problems (C is restored afterwards)
 * and captures the launches in a CUDA graph; run replays the graph on the
 * calling thread's stream and waits for it. */
typedef struct mublis_b200_plan mublis_b200_plan_t;
int mublis_b200_plan_gemm_grouped(char dtype, const mublis_b200_gemm_problem_t *problems,
                                  int count, mublis_b200_plan_t **plan);
int mublis_b200_plan_trsm_grouped(char dtype, const mublis_b200_trsm_problem_t *problems,
                                  int count, mublis_b200_plan_t **plan);
int mublis_b200_plan_run(mublis_b200_plan_t *plan);
int mublis_b200_plan_destroy(mublis_b200_plan_t *plan);

/* Tuned-tile table (the replacement for the reference's compile-time block
 * sizes, targets/<t>/context.c, which a B200 build finds by timing instead).
 * The autotuner's choices (per precision, size class and problem-count
 * bucket) can be kept on disk.  A file is keyed by the GPU (name, SM count,
 * compute capability) and the driver version: loading a file written on
 * another GPU or driver loads nothing.  If MUBLIS_B200_TUNE_FILE names a
 * file, the library loads it at initialisation and rewrites it whenever the
 * autotuner adds a choice.
 *   save:  write the current table to `path` (atomically: temp + rename);
 *   load:  merge `path` into the table, *entries = choices loaded (0 when
 *          the file is missing or keyed to another GPU / driver);
 *   reset: forget every choice (the defaults apply until re-tuned). */
int mublis_b200_tune_save(const char *path);
int mublis_b200_tune_load(const char *path, int *entries);
int mublis_b200_tune_reset(void);

/* ---- request server (no counterpart in the reference) -------------------
 * Continuous batching of Level-3 calls issued by many host threads.  Once a
 * server is attached, every cblas_* / mublis_* call whose operands are ALL
 * device-resident becomes a request: the calling thread blocks until it
 * completes (calls stay synchronous), while the server's scheduler thread
 * coalesces small plain GEMMs (max(m,n,k) <= small_max_dim) and small left
 * TRSMs (order <= 256) waiting together into one grouped launch per
 * precision, and issues the rest asynchronously on a pool of streams,
 * admitting each when its scratch estimate fits the HBM budget.  Calls with
 * host operands keep the direct path.  Creation reserves half the budget
 * (at most half of the free device memory) in CUDA's stream-ordered pool,
 * which keeps it for the process, so that requests never wait for the pool
 * to grow. */
typedef struct {
  size_t hbm_budget_bytes; /* device memory for handles + scratch (0: 64 GiB) */
  int streams;             /* concurrent streams (0: 4) */
  int batch_window_us;     /* extra wait for small arrivals to coalesce (0: none) */
  int small_max_dim;       /* batchable GEMM size limit (0: 512) */
  int max_batch;           /* requests per grouped launch (0: 4096) */
  const char *sform;       /* precision form for non-batched FP32 work (NULL: default) */
  const char *dform;       /* same for FP64 ("plain", "ozaki:8", ...) */
} mublis_b200_server_config_t;

typedef struct {
  unsigned long long completed, batches, batched_requests, queue_depth;
  double p50_latency_s, p99_latency_s, mean_latency_s;
  double tflops;    /* completed flops / (last completion - first submission) */
  double elapsed_s;
  size_t hbm_in_use;
} mublis_b200_server_stats_t;

typedef struct mublis_b200_server mublis_b200_server_t;
int mublis_b200_server_create(const mublis_b200_server_config_t *cfg, mublis_b200_server_t **srv);
int mublis_b200_server_destroy(mublis_b200_server_t *srv);
/* Route this process's device-resident calls through srv (NULL detaches). */
int mublis_b200_server_attach(mublis_b200_server_t *srv);
/* Operand handles: device memory counted against the server's HBM budget
 * (status 3 when it would be exceeded). */
int mublis_b200_server_alloc(mublis_b200_server_t *srv, size_t bytes, void **device_ptr);
int mublis_b200_server_free(mublis_b200_server_t *srv, void *device_ptr);
int mublis_b200_server_stats(mublis_b200_server_t *srv, mublis_b200_server_stats_t *out);
int mublis_b200_server_reset_stats(mublis_b200_server_t *srv);

/* SGEMM that allocates no memory.  No counterpart in the reference (its
 * CPU library draws packing buffers from a host pool, frame/base/pool.c).
 *
 * For callers that cannot allocate device memory when they call in: a
 * process whose GPU memory is already owned by another allocator, or a
 * service that keeps a fixed device footprint and bans cudaMalloc/cudaFree
 * on its request path.  Same arguments, checks and result as mublis_sgemm
 * with the plain FP32 kernel (the form chosen by MUBLIS_B200_SFORM or
 * mublis_b200_set_form does not apply here), but A, B and C must be device
 * pointers (staging host buffers would allocate), and the packed operand
 * panels live in a fixed 32 MiB scratch array in the library's device code.
 * Limit:
 *   (roundup(m, 128) + roundup(n, 128)) * roundup(k, 16) <= 8388608 floats
 * (e.g. m = n = k = 2048); larger sizes return 1 with a message in
 * mublis_b200_last_error() and leave C untouched.
 * The array is claimed once per device: on the device current when the
 * library initialises (mublis_b200_init, or the first call of any entry
 * point), at that point; on any other device, by the first call of this
 * function there, which looks up the array's device address with that
 * device current -- make that first call before any stream capture.  The
 * device keeps the array until the process exits.  All calls on a device
 * share it and it keeps the last call's contents (nothing in it needs to
 * start at zero); calls that overlap on the GPU race on it, so do not
 * overlap them.  Like the other entry points, it returns after
 * synchronizing the calling thread's library stream. */
int mublis_b200_sgemm_noalloc(mublis_trans_t trans_a, mublis_trans_t trans_b, int m, int n, int k,
                              float alpha, const float *a, int rs_a, int cs_a, const float *b,
                              int rs_b, int cs_b, float beta, float *c, int rs_c, int cs_c);

#ifdef __cplusplus
}
#endif

#endif
