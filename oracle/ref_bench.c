/*
 * ref_bench.c -- times a CPU MuBLIS build (the reference's own avx2 or
 * reference config, built into oracle/_ref by this directory's Makefile)
 * through its cblas_* ABI.  Test/benchmark infrastructure only.
 *
 *   ref_bench LIB ROUTINE DTYPE M N K THREADS REPS WARMUP
 *     ROUTINE  gemm_nn gemm_nt gemm_tn gemm_tt symm syrk syr2k trmm trsm
 *              (symm/trmm/trsm: left, lower, non-unit; syrk/syr2k: lower,
 *              no-trans -- the shapes of the plain-family workload), or
 *              "family": all nine in both precisions, one after another
 *              (m = n = k = M), as one timed unit
 *     DTYPE    s | d (ignored for "family")
 *
 * Every thread owns its operands (seeded Philox uniform[-1,1), column-major;
 * TRSM's A has off-diagonals uniform/m and a diagonal in [1,2)) and issues
 * WARMUP untimed, then REPS timed calls; threads start together behind a
 * barrier.  Times come from clock_gettime(CLOCK_MONOTONIC).  Prints one JSON
 * object: per-call median seconds, and aggregate GFLOP/s over the timed
 * region (BLAS-standard flop counts: gemm 2mnk, symm 2m^2n, syrk n(n+1)k,
 * syr2k 2n(n+1)k, trmm m^2n, trsm m^2n).
 */
#include <dlfcn.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "philox.h"

enum { ROW = 101, COL = 102, NT = 111, TR = 112, UP = 121, LO = 122, NU = 131, LEFT = 141 };

typedef void (*gemm_s_t)(int, int, int, int, int, int, float, const float *, int, const float *, int, float, float *, int);
typedef void (*gemm_d_t)(int, int, int, int, int, int, double, const double *, int, const double *, int, double, double *, int);
typedef void (*symm_s_t)(int, int, int, int, int, float, const float *, int, const float *, int, float, float *, int);
typedef void (*symm_d_t)(int, int, int, int, int, double, const double *, int, const double *, int, double, double *, int);
typedef void (*syrk_s_t)(int, int, int, int, int, float, const float *, int, float, float *, int);
typedef void (*syrk_d_t)(int, int, int, int, int, double, const double *, int, double, double *, int);
typedef void (*tr_s_t)(int, int, int, int, int, int, int, float, const float *, int, float *, int);
typedef void (*tr_d_t)(int, int, int, int, int, int, int, double, const double *, int, double *, int);

static void *g_lib;
static const char *g_routine;
static int g_dbl, g_m, g_n, g_k, g_threads, g_reps, g_warmup;
static const char *FAMILY[] = {"gemm_nn", "gemm_nt", "gemm_tn", "gemm_tt", "symm",
                               "syrk",    "syr2k",   "trmm",    "trsm"};
static pthread_barrier_t g_start, g_done;
static double *g_times;

static double now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void *sym(const char *name) {
  void *f = dlsym(g_lib, name);
  if (!f) { fprintf(stderr, "missing symbol %s\n", name); exit(2); }
  return f;
}

static void fill(int dbl, void *x, long m, long n, uint32_t id, int trsm_a) {
  for (long j = 0; j < n; ++j)
    for (long i = 0; i < m; ++i) {
      uint64_t idx = (uint64_t)(i + j * m);
      double v;
      if (trsm_a && i == j) v = dbl ? philox_draw_f64(idx, 0, id, PHILOX_DRAW_DIAG)
                                       : philox_draw_f32(idx, 0, id, PHILOX_DRAW_DIAG);
      else {
        v = dbl ? philox_draw_f64(idx, 0, id, PHILOX_DRAW_UNIFORM)
                  : philox_draw_f32(idx, 0, id, PHILOX_DRAW_UNIFORM);
        if (trsm_a) v /= (double)m;
      }
      if (dbl) ((double *)x)[i + j * m] = v;
      else ((float *)x)[i + j * m] = (float)v;
    }
}

static void call_once(const char *r, int dbl, void *a, void *b, void *c) {
  int m = g_m, n = g_n, k = g_k;
  double al = 0.75, be = 0.25;
  if (!strncmp(r, "gemm_", 5)) {
    int ta = r[5] == 't' ? TR : NT, tb = r[6] == 't' ? TR : NT;
    int lda = ta == NT ? m : k, ldb = tb == NT ? k : n;
    if (dbl) ((gemm_d_t)sym("cblas_dgemm"))(COL, ta, tb, m, n, k, al, a, lda, b, ldb, be, c, m);
    else ((gemm_s_t)sym("cblas_sgemm"))(COL, ta, tb, m, n, k, (float)al, a, lda, b, ldb, (float)be, c, m);
  } else if (!strcmp(r, "symm")) {
    if (dbl) ((symm_d_t)sym("cblas_dsymm"))(COL, LEFT, LO, m, n, al, a, m, b, m, be, c, m);
    else ((symm_s_t)sym("cblas_ssymm"))(COL, LEFT, LO, m, n, (float)al, a, m, b, m, (float)be, c, m);
  } else if (!strcmp(r, "syrk")) {
    if (dbl) ((syrk_d_t)sym("cblas_dsyrk"))(COL, LO, NT, n, k, al, a, n, be, c, n);
    else ((syrk_s_t)sym("cblas_ssyrk"))(COL, LO, NT, n, k, (float)al, a, n, (float)be, c, n);
  } else if (!strcmp(r, "syr2k")) {
    if (dbl) ((symm_d_t)sym("cblas_dsyr2k"))(COL, LO, NT, n, k, al, a, n, b, n, be, c, n);
    else ((symm_s_t)sym("cblas_ssyr2k"))(COL, LO, NT, n, k, (float)al, a, n, b, n, (float)be, c, n);
  } else if (!strcmp(r, "trmm") || !strcmp(r, "trsm")) {
    const char *name = dbl ? (r[2] == 'm' ? "cblas_dtrmm" : "cblas_dtrsm")
                             : (r[2] == 'm' ? "cblas_strmm" : "cblas_strsm");
    if (dbl) ((tr_d_t)sym(name))(COL, LEFT, LO, NT, NU, m, n, al, a, m, c, m);
    else ((tr_s_t)sym(name))(COL, LEFT, LO, NT, NU, m, n, (float)al, a, m, c, m);
  } else {
    fprintf(stderr, "unknown routine %s\n", r);
    exit(2);
  }
}

typedef struct {
  const char *routine;
  int dbl;
  void *a, *b, *c, *c0;
  size_t cbytes;
} op_t;

static void setup(op_t *op) {
  size_t es = op->dbl ? 8 : 4;
  long m = g_m, n = g_n, k = g_k;
  long arows = m, acols = k, brows = k, bcols = n, crows = m, ccols = n;
  const char *r = op->routine;
  if (!strcmp(r, "symm") || !strncmp(r, "tr", 2)) { acols = m; brows = m; }
  if (!strncmp(r, "syr", 3)) { arows = n; acols = k; brows = n; bcols = k; crows = n; ccols = n; }
  if (!strncmp(r, "gemm_", 5)) {
    if (r[5] == 't') { arows = k; acols = m; }
    if (r[6] == 't') { brows = n; bcols = k; }
  }
  op->a = malloc(es * arows * acols);
  op->b = malloc(es * brows * bcols);
  op->c = malloc(es * crows * ccols);
  op->c0 = malloc(es * crows * ccols);
  op->cbytes = es * crows * ccols;
  fill(op->dbl, op->a, arows, acols, 0, !strcmp(r, "trsm"));
  fill(op->dbl, op->b, brows, bcols, 1, 0);
  fill(op->dbl, op->c0, crows, ccols, 2, 0);
}

static void run_op(op_t *op) {
  memcpy(op->c, op->c0, op->cbytes);
  call_once(op->routine, op->dbl, op->a, op->b, op->c);
}

static void *worker(void *vp) {
  long t = (long)vp;
  int family = !strcmp(g_routine, "family");
  int nops = family ? 18 : 1;
  op_t ops[18];
  for (int q = 0; q < nops; ++q) {
    ops[q].routine = family ? FAMILY[q % 9] : g_routine;
    ops[q].dbl = family ? q >= 9 : g_dbl;
    setup(&ops[q]);
  }
  for (int w = 0; w < g_warmup; ++w)
    for (int q = 0; q < nops; ++q) run_op(&ops[q]);
  pthread_barrier_wait(&g_start);
  for (int r = 0; r < g_reps; ++r) {
    double t0 = now();
    for (int q = 0; q < nops; ++q) run_op(&ops[q]);
    g_times[t * g_reps + r] = now() - t0;
  }
  pthread_barrier_wait(&g_done);
  for (int q = 0; q < nops; ++q) {
    free(ops[q].a); free(ops[q].b); free(ops[q].c); free(ops[q].c0);
  }
  return NULL;
}

static double flops_of(const char *r, double m, double n, double k) {
  if (!strncmp(r, "gemm", 4)) return 2 * m * n * k;
  if (!strcmp(r, "symm")) return 2 * m * m * n;
  if (!strcmp(r, "syrk")) return n * (n + 1) * k;
  if (!strcmp(r, "syr2k")) return 2 * n * (n + 1) * k;
  return m * m * n;
}

static int cmp(const void *x, const void *y) {
  double a = *(const double *)x, b = *(const double *)y;
  return (a > b) - (a < b);
}

int main(int argc, char **argv) {
  if (argc < 10) {
    fprintf(stderr, "usage: %s LIB ROUTINE DTYPE M N K THREADS REPS WARMUP\n", argv[0]);
    return 2;
  }
  g_lib = dlopen(argv[1], RTLD_NOW | RTLD_LOCAL);
  if (!g_lib) { fprintf(stderr, "%s\n", dlerror()); return 2; }
  g_routine = argv[2];
  g_dbl = argv[3][0] == 'd';
  g_m = atoi(argv[4]); g_n = atoi(argv[5]); g_k = atoi(argv[6]);
  g_threads = atoi(argv[7]); g_reps = atoi(argv[8]); g_warmup = atoi(argv[9]);
  if (g_threads < 1 || g_reps < 1) return 2;
  g_times = calloc((size_t)g_threads * g_reps, sizeof(double));
  pthread_barrier_init(&g_start, NULL, (unsigned)g_threads + 1);
  pthread_barrier_init(&g_done, NULL, (unsigned)g_threads + 1);
  pthread_t *tid = malloc(sizeof(pthread_t) * g_threads);
  for (long t = 0; t < g_threads; ++t) pthread_create(&tid[t], NULL, worker, (void *)t);
  pthread_barrier_wait(&g_start);
  double t0 = now();
  pthread_barrier_wait(&g_done);
  double wall = now() - t0;
  for (int t = 0; t < g_threads; ++t) pthread_join(tid[t], NULL);

  double flops = 0;
  const char *r = g_routine;
  if (!strcmp(r, "family"))
    for (int q = 0; q < 18; ++q) flops += flops_of(FAMILY[q % 9], g_m, g_n, g_k);
  else
    flops = flops_of(r, g_m, g_n, g_k);
  int total = g_threads * g_reps;
  qsort(g_times, (size_t)total, sizeof(double), cmp);
  double median = g_times[total / 2];
  printf("{\"routine\": \"%s\", \"dtype\": \"%c\", \"m\": %d, \"n\": %d, \"k\": %d, "
         "\"threads\": %d, \"reps\": %d, \"median_s\": %.6g, \"wall_s\": %.6g, "
         "\"flops_per_call\": %.6g, \"gflops_per_thread\": %.6g, \"gflops_aggregate\": %.6g}\n",
         r, argv[3][0], g_m, g_n, g_k, g_threads, g_reps, median, wall, flops,
         flops / median * 1e-9, flops * total / wall * 1e-9);
  return 0;
}
