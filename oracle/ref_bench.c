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
 *     DTYPE    s | d (ignored for "family" and "family_par")
 *     ROUTINE "family_par": the same 18 calls at m = n = k = M, each step
 *              spread over all THREADS: every call is cut into column panels
 *              of PANEL columns (argument 10, default 512) that are separate
 *              cblas calls of the reference library (GEMM / SYMM / TRMM /
 *              TRSM: the panel's columns of C or B; SYRK / SYR2K: the
 *              panel's diagonal block as a SYRK / SYR2K plus the rows below
 *              it as GEMMs), so a single-threaded library fills every host
 *              thread.  The panels' flops add up to the whole calls' flops.
 *              Threads take panels largest first from a shared queue; one
 *              step is one pass over all of them.  Operands are shared by
 *              the threads (one set, seed 0, matrix ids 3c + {0, 1, 2} for
 *              call c, as the GPU benchmark builds them; TRMM and TRSM get
 *              the TRSM operand).  A negative PANEL checks the panels
 *              against whole calls instead of timing them.
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

/* ---- family_par: one shared operand set, column panels over all threads -- */

typedef struct {
  int call; /* 0..17: the family call the panel belongs to */
  int kind; /* 0 gemm, 1 symm, 2 syrk, 3 syr2k, 4 trmm, 5 trsm */
  int dbl, ta, tb;
  long j0, w; /* panel columns [j0, j0 + w) */
  double flops;
  void *a, *b, *c;
} task_t;

static task_t *g_tasks;
static int g_ntasks;
static volatile int g_next;
static pthread_mutex_t g_next_mu = PTHREAD_MUTEX_INITIALIZER;

static int take_task(void) {
  pthread_mutex_lock(&g_next_mu);
  int t = g_next < g_ntasks ? g_next++ : -1;
  pthread_mutex_unlock(&g_next_mu);
  return t;
}

#define ELT(dbl, p, off) ((void *)((char *)(p) + (size_t)(off) * ((dbl) ? 8 : 4)))

static void run_task(const task_t *t) {
  const long n = g_m, j0 = t->j0, w = t->w, j1 = j0 + w;
  const double al = 0.75, be = 0.25;
  const int d = t->dbl;
  gemm_d_t dg = (gemm_d_t)sym("cblas_dgemm");
  gemm_s_t sg = (gemm_s_t)sym("cblas_sgemm");
#define GEMM(ta, tb, m_, n_, k_, A, lda, B, ldb, beta, C)                                       \
  do {                                                                                        \
    if (d) dg(COL, ta, tb, (int)(m_), (int)(n_), (int)(k_), al, A, (int)(lda), B, (int)(ldb), \
              beta, C, (int)n);                                                               \
    else sg(COL, ta, tb, (int)(m_), (int)(n_), (int)(k_), (float)al, A, (int)(lda), B,        \
            (int)(ldb), (float)(beta), C, (int)n);                                            \
  } while (0)
  switch (t->kind) {
  case 0: { /* C[:, J] = al op(A) op(B)[:, J] + be C[:, J] */
    void *bj = t->tb == NT ? ELT(d, t->b, j0 * n) : ELT(d, t->b, j0);
    GEMM(t->ta, t->tb, n, w, n, t->a, n, bj, n, be, ELT(d, t->c, j0 * n));
    break;
  }
  case 1:
    if (d) ((symm_d_t)sym("cblas_dsymm"))(COL, LEFT, LO, (int)n, (int)w, al, t->a, (int)n,
                                          ELT(d, t->b, j0 * n), (int)n, be,
                                          ELT(d, t->c, j0 * n), (int)n);
    else ((symm_s_t)sym("cblas_ssymm"))(COL, LEFT, LO, (int)n, (int)w, (float)al, t->a, (int)n,
                                        ELT(d, t->b, j0 * n), (int)n, (float)be,
                                        ELT(d, t->c, j0 * n), (int)n);
    break;
  case 2: /* C[J, J] lower by SYRK; C[j1:, J] = al A[j1:, :] A[J, :]^T + be C[j1:, J] */
    if (d) ((syrk_d_t)sym("cblas_dsyrk"))(COL, LO, NT, (int)w, (int)n, al, ELT(d, t->a, j0),
                                          (int)n, be, ELT(d, t->c, j0 + j0 * n), (int)n);
    else ((syrk_s_t)sym("cblas_ssyrk"))(COL, LO, NT, (int)w, (int)n, (float)al,
                                        ELT(d, t->a, j0), (int)n, (float)be,
                                        ELT(d, t->c, j0 + j0 * n), (int)n);
    if (j1 < n)
      GEMM(NT, TR, n - j1, w, n, ELT(d, t->a, j1), n, ELT(d, t->a, j0), n, be,
           ELT(d, t->c, j1 + j0 * n));
    break;
  case 3: /* SYR2K diagonal block, then both products below it */
    if (d) ((symm_d_t)sym("cblas_dsyr2k"))(COL, LO, NT, (int)w, (int)n, al, ELT(d, t->a, j0),
                                           (int)n, ELT(d, t->b, j0), (int)n, be,
                                           ELT(d, t->c, j0 + j0 * n), (int)n);
    else ((symm_s_t)sym("cblas_ssyr2k"))(COL, LO, NT, (int)w, (int)n, (float)al,
                                         ELT(d, t->a, j0), (int)n, ELT(d, t->b, j0), (int)n,
                                         (float)be, ELT(d, t->c, j0 + j0 * n), (int)n);
    if (j1 < n) {
      GEMM(NT, TR, n - j1, w, n, ELT(d, t->a, j1), n, ELT(d, t->b, j0), n, be,
           ELT(d, t->c, j1 + j0 * n));
      GEMM(NT, TR, n - j1, w, n, ELT(d, t->b, j1), n, ELT(d, t->a, j0), n, 1.0,
           ELT(d, t->c, j1 + j0 * n));
    }
    break;
  default: {
    const char *name = d ? (t->kind == 4 ? "cblas_dtrmm" : "cblas_dtrsm")
                         : (t->kind == 4 ? "cblas_strmm" : "cblas_strsm");
    if (d) ((tr_d_t)sym(name))(COL, LEFT, LO, NT, NU, (int)n, (int)w, al, t->a, (int)n,
                               ELT(d, t->b, j0 * n), (int)n);
    else ((tr_s_t)sym(name))(COL, LEFT, LO, NT, NU, (int)n, (int)w, (float)al, t->a, (int)n,
                             ELT(d, t->b, j0 * n), (int)n);
  }
  }
#undef GEMM
}

typedef struct {
  void *x;
  int dbl;
  long n;
  uint32_t id;
  int tri; /* TRSM operand: off-diagonals uniform / n, diagonal in [1, 2) */
} fill_job_t;

static fill_job_t g_fills[64];
static int g_nfills;
static volatile int g_next_fill;

static void *fill_worker(void *vp) {
  (void)vp;
  for (;;) {
    pthread_mutex_lock(&g_next_mu);
    int f = g_next_fill < g_nfills ? g_next_fill++ : -1;
    pthread_mutex_unlock(&g_next_mu);
    if (f < 0) return NULL;
    fill(g_fills[f].dbl, g_fills[f].x, g_fills[f].n, g_fills[f].n, g_fills[f].id, g_fills[f].tri);
  }
}

static pthread_barrier_t g_step_start, g_step_done;
static volatile int g_quit;

static void *par_worker(void *vp) {
  (void)vp;
  for (;;) {
    pthread_barrier_wait(&g_step_start);
    if (g_quit) return NULL;
    for (int t; (t = take_task()) >= 0;) run_task(&g_tasks[t]);
    pthread_barrier_wait(&g_step_done);
  }
}

static int cmp_task(const void *x, const void *y) {
  double a = ((const task_t *)x)->flops, b = ((const task_t *)y)->flops;
  return (a < b) - (a > b); /* largest first */
}

static int family_par(long n, int threads, int reps, int warmup, long panel, int check) {
  void *ops[18][3];
  g_nfills = 0;
  for (int c = 0; c < 18; ++c) {
    const int dbl = c >= 9, kind = c % 9;
    const size_t bytes = (size_t)n * n * (dbl ? 8 : 4);
    for (int i = 0; i < 3; ++i) {
      ops[c][i] = NULL;
      if (i == 2 && kind >= 7) continue; /* TRMM / TRSM: B is the in/out operand */
      ops[c][i] = malloc(bytes);
      if (!ops[c][i]) { fprintf(stderr, "out of host memory\n"); return 2; }
      g_fills[g_nfills++] = (fill_job_t){ops[c][i], dbl, n, (uint32_t)(3 * c + i),
                                         i == 0 && kind >= 7};
    }
  }
  g_next_fill = 0;
  pthread_t *tid = malloc(sizeof(pthread_t) * threads);
  for (int t = 0; t < threads; ++t) pthread_create(&tid[t], NULL, fill_worker, NULL);
  for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);

  g_tasks = malloc(sizeof(task_t) * 18 * (n / panel + 1));
  g_ntasks = 0;
  double step_flops = 0;
  for (int c = 0; c < 18; ++c) {
    const int dbl = c >= 9, r = c % 9;
    for (long j0 = 0; j0 < n; j0 += panel) {
      task_t t;
      memset(&t, 0, sizeof t);
      t.call = c;
      t.dbl = dbl;
      t.j0 = j0;
      t.w = j0 + panel <= n ? panel : n - j0;
      t.a = ops[c][0];
      t.b = ops[c][1];
      t.c = ops[c][2];
      const double w = (double)t.w, N = (double)n, below = N - (double)(j0 + t.w);
      if (r < 4) {
        t.kind = 0;
        t.ta = FAMILY[r][5] == 't' ? TR : NT;
        t.tb = FAMILY[r][6] == 't' ? TR : NT;
        t.flops = 2 * N * w * N;
      } else if (r == 4) {
        t.kind = 1;
        t.flops = 2 * N * N * w;
      } else if (r == 5) {
        t.kind = 2;
        t.flops = w * (w + 1) * N + 2 * below * w * N;
      } else if (r == 6) {
        t.kind = 3;
        t.flops = 2 * w * (w + 1) * N + 4 * below * w * N;
      } else {
        t.kind = r == 7 ? 4 : 5;
        t.flops = N * N * w;
      }
      step_flops += t.flops;
      g_tasks[g_ntasks++] = t;
    }
  }
  qsort(g_tasks, (size_t)g_ntasks, sizeof(task_t), cmp_task);

  if (check) {
    /* Check mode: the panels of one pass against each call made whole on
     * copies of the same inputs; prints the largest normwise difference
     * ||C_panels - C_whole||_F / ||C_whole||_F over the 18 calls. */
    double worst = 0;
    void *outs[18], *whole[18];
    for (int c = 0; c < 18; ++c) {
      const int dbl = c >= 9, io = c % 9 >= 7 ? 1 : 2;
      const size_t bytes = (size_t)n * n * (dbl ? 8 : 4);
      whole[c] = malloc(bytes);
      memcpy(whole[c], ops[c][io], bytes);
      outs[c] = ops[c][io];
    }
    for (int t = 0; t < g_ntasks; ++t) run_task(&g_tasks[t]);
    const long gm = g_m;
    for (int c = 0; c < 18; ++c) {
      const int dbl = c >= 9, io = c % 9 >= 7 ? 1 : 2;
      task_t t = g_tasks[0];
      for (int q = 0; q < g_ntasks; ++q)
        if (g_tasks[q].call == c) {
          t = g_tasks[q];
          break;
        }
      t.j0 = 0;
      t.w = gm;
      if (io == 1) t.b = whole[c]; else t.c = whole[c];
      run_task(&t);
      double num = 0, den = 0;
      for (size_t e = 0; e < (size_t)n * n; ++e) {
        const long i = (long)(e % (size_t)n), j = (long)(e / (size_t)n);
        if ((c % 9 == 5 || c % 9 == 6) && i < j) continue; /* SYRK / SYR2K: lower only */
        double x = dbl ? ((double *)outs[c])[e] : ((float *)outs[c])[e];
        double y = dbl ? ((double *)whole[c])[e] : ((float *)whole[c])[e];
        num += (x - y) * (x - y);
        den += y * y;
      }
      const double rel = den > 0 ? __builtin_sqrt(num / den) : __builtin_sqrt(num);
      if (rel > worst) worst = rel;
      free(whole[c]);
    }
    printf("{\"routine\": \"family_par_check\", \"n\": %ld, \"panel\": %ld, \"tasks\": %d, "
           "\"max_rel_diff\": %.6g}\n", n, panel, g_ntasks, worst);
    for (int c = 0; c < 18; ++c)
      for (int i = 0; i < 3; ++i) free(ops[c][i]);
    free(g_tasks);
    free(tid);
    return 0;
  }

  pthread_barrier_init(&g_step_start, NULL, (unsigned)threads + 1);
  pthread_barrier_init(&g_step_done, NULL, (unsigned)threads + 1);
  g_quit = 0;
  for (int t = 0; t < threads; ++t) pthread_create(&tid[t], NULL, par_worker, NULL);
  double *times = calloc((size_t)reps, sizeof(double));
  double timed = 0;
  for (int s = 0; s < warmup + reps; ++s) {
    g_next = 0;
    double t0 = now();
    pthread_barrier_wait(&g_step_start);
    pthread_barrier_wait(&g_step_done);
    double dt = now() - t0;
    if (s >= warmup) {
      times[s - warmup] = dt;
      timed += dt;
    }
  }
  g_quit = 1;
  pthread_barrier_wait(&g_step_start);
  for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
  qsort(times, (size_t)reps, sizeof(double), cmp);
  printf("{\"routine\": \"family_par\", \"m\": %ld, \"n\": %ld, \"k\": %ld, \"threads\": %d, "
         "\"reps\": %d, \"warmup\": %d, \"panel\": %ld, \"tasks\": %d, \"median_s\": %.6g, "
         "\"wall_s\": %.6g, \"flops_per_step\": %.6g, \"gflops_aggregate\": %.6g}\n",
         n, n, n, threads, reps, warmup, panel, g_ntasks, times[reps / 2], timed, step_flops,
         step_flops * reps / timed * 1e-9);
  for (int c = 0; c < 18; ++c)
    for (int i = 0; i < 3; ++i) free(ops[c][i]);
  free(g_tasks);
  free(times);
  free(tid);
  return 0;
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
  if (!strcmp(g_routine, "family_par")) {
    /* A negative PANEL selects the check mode with panels of -PANEL columns. */
    long panel = argc > 10 ? atol(argv[10]) : 512;
    const int check = panel < 0;
    if (check) panel = -panel;
    if (panel < 1 || g_m < 1 || g_m != g_n || g_m != g_k) return 2;
    return family_par(g_m, g_threads, g_reps, g_warmup, panel, check);
  }
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
