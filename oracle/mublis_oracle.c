/*
 * mublis_oracle.c -- CPU restatement of the reference's Level-3 semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the tests, smoke() and
 * the benchmark's CPU-baseline leg compare the B200 library against; nothing
 * in the product links or calls it.
 *
 * It restates, element by element, what the reference computes:
 *   operand views      frame/l1m/packm.c:4-15 (stored triangle test) and
 *                      :18-84 (general / symmetric reflection / triangular
 *                      zero, unit and inverted diagonal)
 *   generic driver     frame/l3/l3_driver.c:49-249 (domain relations jp, ji,
 *                      pi from frame/l3/l3_utils.c:18-28; beta pass for tiles
 *                      without an update :88-121; beta == 0 never reads C
 *                      :111-112, :224-225; alpha == 0 scales by beta only
 *                      :104, :123)
 *   BLAS shims         frame/l3/gemm.c:14-52, symm.c:14-56, syrk.c:19-51,
 *                      syr2k.c:47-68 (two driver passes, the second with
 *                      beta = 1)
 *   TRMM               frame/l3/trmm.c:44-85 (trans -> stride swap + flipped
 *                      uplo; triangular operand with unit diagonal), :138-144
 *                      (alpha == 0 zeroes B)
 *   TRSM               frame/l3/trsm.c:24-54 (alpha == 0 zeroes B; right ->
 *                      left by swapping m/n and B's strides and toggling
 *                      trans; trans -> stride swap + flipped uplo), :83-85
 *                      with packm.c:143-144 (the diagonal is inverted once in
 *                      working precision and multiplied, never divided)
 *
 * Sums are accumulated in long double (x87, 64-bit significand), so the
 * oracle is more accurate than either the reference or the GPU; parity is a
 * normwise tolerance, not bit equality, because the reference's own result
 * depends on its micro-kernel's summation order.
 *
 * Also here: a double-double (Ogita-Rump-Oishi Dot2: TwoSum + FMA-based
 * TwoProd) evaluator of selected GEMM entries for error studies, and the
 * Philox fills shared with the tests.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/mublis.h"
#include "philox.h"

typedef long double acc_t;

static int g_threads = 1;
void oracle_set_threads(int threads) { g_threads = threads < 1 ? 1 : threads; }

/* frame/l3/l3_utils.c:18-28: LOWER means lhs <= rhs, UPPER lhs >= rhs. */
static int relation_holds(mublis_l3_relation_t rel, long lhs, long rhs) {
  if (rel == MUBLIS_L3_LOWER) return lhs <= rhs;
  if (rel == MUBLIS_L3_UPPER) return lhs >= rhs;
  return 1;
}

/* frame/l1m/packm.c:4-15: is (row - col) inside the stored triangle? */
static int is_stored(mublis_uplo_t uplo, long delta) {
  if (uplo == MUBLIS_LOWER) return delta >= 0;
  if (uplo == MUBLIS_UPPER) return delta <= 0;
  return 1;
}

static mublis_uplo_t flip_uplo(mublis_uplo_t u) {
  return u == MUBLIS_LOWER ? MUBLIS_UPPER : (u == MUBLIS_UPPER ? MUBLIS_LOWER : MUBLIS_DENSE);
}

/* Logical element (r, c) of a stored operand, following packm.c:40-71.  For
 * the A operand (r, c) = (i, p); for the B operand (r, c) = (p, j) -- the
 * reference packs B with swapped strides and flip_uplo(uplo), which yields
 * the same stored-triangle test on (p - j).  Returns 0 for "structural zero"
 * and never touches memory outside the stored triangle. */
#define DEFINE_ELEM(ctype, suffix)                                                       \
  static acc_t elem_##suffix(const ctype *x, long rs, long cs,                           \
                             const mublis_l3_operand_t *op, long r, long c) {            \
    long delta = r - c;                                                                  \
    switch (op->struc) {                                                                 \
    case MUBLIS_STRUC_SYMMETRIC:                                                         \
      if (is_stored(op->uplo, delta)) return (acc_t)x[r * rs + c * cs];                  \
      return (acc_t)x[c * rs + r * cs];                                                  \
    case MUBLIS_STRUC_TRIANGULAR:                                                        \
      if (!is_stored(op->uplo, delta)) return 0;                                         \
      if (delta == 0 && op->diag == MUBLIS_PACKM_DIAG_UNIT) return 1;                    \
      if (delta == 0 && op->diag == MUBLIS_PACKM_DIAG_INVERT)                            \
        return (acc_t)((ctype)1 / x[r * rs + c * cs]);                                   \
      return (acc_t)x[r * rs + c * cs];                                                  \
    default:                                                                             \
      return (acc_t)x[r * rs + c * cs];                                                  \
    }                                                                                    \
  }
DEFINE_ELEM(float, s)
DEFINE_ELEM(double, d)

/* ---- generic driver (l3_driver.c:49-249), element-wise ------------------ */

#define DEFINE_DRIVER(ctype, suffix)                                                     \
  typedef struct {                                                                       \
    int m, n, k;                                                                         \
    ctype alpha, beta;                                                                   \
    const ctype *a; long rs_a, cs_a;                                                     \
    const ctype *b; long rs_b, cs_b;                                                     \
    ctype *c; long rs_c, cs_c;                                                           \
    const mublis_l3_product_t *pr;                                                       \
    int j0, j1;                                                                          \
  } drv_args_##suffix;                                                                   \
                                                                                         \
  static void *driver_cols_##suffix(void *vp) {                                          \
    drv_args_##suffix *g = (drv_args_##suffix *)vp;                                      \
    const mublis_l3_domain_t dom = g->pr->domain;                                        \
    acc_t *acc = (acc_t *)malloc(sizeof(acc_t) * (size_t)(g->m > 0 ? g->m : 1));         \
    for (long j = g->j0; j < g->j1; ++j) {                                               \
      for (long i = 0; i < g->m; ++i) acc[i] = 0;                                        \
      if (g->alpha != (ctype)0) {                                                        \
        for (long p = 0; p < g->k; ++p) {                                                \
          if (!relation_holds(dom.jp, j, p)) continue;                                   \
          acc_t bpj = elem_##suffix(g->b, g->rs_b, g->cs_b, &g->pr->b, p, j);            \
          for (long i = 0; i < g->m; ++i) {                                              \
            if (!relation_holds(dom.pi, p, i)) continue;                                 \
            if (!relation_holds(dom.ji, j, i)) continue;                                 \
            acc[i] += elem_##suffix(g->a, g->rs_a, g->cs_a, &g->pr->a, i, p) * bpj;      \
          }                                                                              \
        }                                                                                \
      }                                                                                  \
      for (long i = 0; i < g->m; ++i) {                                                  \
        if (!relation_holds(dom.ji, j, i)) continue;                                     \
        ctype *cij = &g->c[i * g->rs_c + j * g->cs_c];                                   \
        acc_t v = g->alpha != (ctype)0 ? (acc_t)g->alpha * acc[i] : 0;                   \
        if (g->beta != (ctype)0) v += (acc_t)g->beta * (acc_t)(*cij);                    \
        *cij = (ctype)v;                                                                 \
      }                                                                                  \
    }                                                                                    \
    free(acc);                                                                           \
    return NULL;                                                                         \
  }                                                                                      \
                                                                                         \
  int oracle_l3_##suffix##driver(int m, int n, int k, ctype alpha, const ctype *a,       \
                                 int rs_a, int cs_a, const ctype *b, int rs_b, int cs_b, \
                                 ctype beta, ctype *c, int rs_c, int cs_c,               \
                                 const mublis_l3_product_t *product) {                   \
    if (m == 0 || n == 0) return 0;                                                      \
    int t = g_threads < n ? g_threads : n;                                               \
    pthread_t tid[256];                                                                  \
    drv_args_##suffix args[256];                                                         \
    if (t > 256) t = 256;                                                                \
    for (int q = 0; q < t; ++q) {                                                        \
      drv_args_##suffix g = {m, n, k, alpha, beta, a, rs_a, cs_a, b, rs_b, cs_b,         \
                             c, rs_c, cs_c, product,                                     \
                             (int)((long)n * q / t), (int)((long)n * (q + 1) / t)};      \
      args[q] = g;                                                                       \
    }                                                                                    \
    if (t == 1) { driver_cols_##suffix(&args[0]); return 0; }                            \
    for (int q = 0; q < t; ++q) pthread_create(&tid[q], NULL, driver_cols_##suffix, &args[q]); \
    for (int q = 0; q < t; ++q) pthread_join(tid[q], NULL);                              \
    return 0;                                                                            \
  }
DEFINE_DRIVER(float, s)
DEFINE_DRIVER(double, d)

static const mublis_l3_operand_t OP_GENERAL = {MUBLIS_STRUC_GENERAL, MUBLIS_DENSE,
                                               MUBLIS_PACKM_DIAG_NONUNIT};

static mublis_l3_relation_t uplo_relation(mublis_uplo_t u) {
  return u == MUBLIS_LOWER ? MUBLIS_L3_LOWER : (u == MUBLIS_UPPER ? MUBLIS_L3_UPPER : MUBLIS_L3_ALL);
}

/* ---- BLAS shims --------------------------------------------------------- */

#define DEFINE_SHIMS(ctype, s)                                                           \
  /* frame/l3/gemm.c:14-52 */                                                            \
  int oracle_##s##gemm(mublis_trans_t ta, mublis_trans_t tb, int m, int n, int k,        \
                       ctype alpha, const ctype *a, int rs_a, int cs_a, const ctype *b,  \
                       int rs_b, int cs_b, ctype beta, ctype *c, int rs_c, int cs_c) {   \
    if (ta == MUBLIS_TRANSPOSE) { int t = rs_a; rs_a = cs_a; cs_a = t; }                 \
    if (tb == MUBLIS_TRANSPOSE) { int t = rs_b; rs_b = cs_b; cs_b = t; }                 \
    mublis_l3_product_t pr = {{MUBLIS_L3_ALL, MUBLIS_L3_ALL, MUBLIS_L3_ALL},             \
                              OP_GENERAL, OP_GENERAL};                                   \
    return oracle_l3_##s##driver(m, n, k, alpha, a, rs_a, cs_a, b, rs_b, cs_b, beta, c,  \
                                 rs_c, cs_c, &pr);                                       \
  }                                                                                      \
  /* frame/l3/symm.c:14-56: left -> A symmetric, k = m; right -> roles swap */           \
  int oracle_##s##symm(mublis_side_t side, mublis_uplo_t uplo, int m, int n,             \
                       ctype alpha, const ctype *a, int rs_a, int cs_a, const ctype *b,  \
                       int rs_b, int cs_b, ctype beta, ctype *c, int rs_c, int cs_c) {   \
    mublis_l3_operand_t sym = {MUBLIS_STRUC_SYMMETRIC, uplo, MUBLIS_PACKM_DIAG_NONUNIT};  \
    mublis_l3_product_t pr = {{MUBLIS_L3_ALL, MUBLIS_L3_ALL, MUBLIS_L3_ALL},             \
                              side == MUBLIS_LEFT ? sym : OP_GENERAL,                    \
                              side == MUBLIS_RIGHT ? sym : OP_GENERAL};                  \
    if (side == MUBLIS_LEFT)                                                             \
      return oracle_l3_##s##driver(m, n, m, alpha, a, rs_a, cs_a, b, rs_b, cs_b, beta,   \
                                   c, rs_c, cs_c, &pr);                                  \
    return oracle_l3_##s##driver(m, n, n, alpha, b, rs_b, cs_b, a, rs_a, cs_a, beta, c,  \
                                 rs_c, cs_c, &pr);                                       \
  }                                                                                      \
  /* frame/l3/syrk.c:19-51: ji selects the triangle, B = A with swapped strides */       \
  int oracle_##s##syrk(mublis_uplo_t uplo, mublis_trans_t trans, int n, int k,           \
                       ctype alpha, const ctype *a, int rs_a, int cs_a, ctype beta,      \
                       ctype *c, int rs_c, int cs_c) {                                   \
    if (trans == MUBLIS_TRANSPOSE) { int t = rs_a; rs_a = cs_a; cs_a = t; }              \
    mublis_l3_product_t pr = {{MUBLIS_L3_ALL, uplo_relation(uplo), MUBLIS_L3_ALL},       \
                              OP_GENERAL, OP_GENERAL};                                   \
    return oracle_l3_##s##driver(n, n, k, alpha, a, rs_a, cs_a, a, cs_a, rs_a, beta, c,  \
                                 rs_c, cs_c, &pr);                                       \
  }                                                                                      \
  /* frame/l3/syr2k.c:47-68: two passes, the second with beta = 1 */                     \
  int oracle_##s##syr2k(mublis_uplo_t uplo, mublis_trans_t trans, int n, int k,          \
                        ctype alpha, const ctype *a, int rs_a, int cs_a, const ctype *b, \
                        int rs_b, int cs_b, ctype beta, ctype *c, int rs_c, int cs_c) {  \
    if (trans == MUBLIS_TRANSPOSE) {                                                     \
      int t = rs_a; rs_a = cs_a; cs_a = t;                                               \
      t = rs_b; rs_b = cs_b; cs_b = t;                                                   \
    }                                                                                    \
    mublis_l3_product_t pr = {{MUBLIS_L3_ALL, uplo_relation(uplo), MUBLIS_L3_ALL},       \
                              OP_GENERAL, OP_GENERAL};                                   \
    int st = oracle_l3_##s##driver(n, n, k, alpha, a, rs_a, cs_a, b, cs_b, rs_b, beta,   \
                                   c, rs_c, cs_c, &pr);                                  \
    if (st) return st;                                                                   \
    return oracle_l3_##s##driver(n, n, k, alpha, b, rs_b, cs_b, a, cs_a, rs_a,           \
                                 (ctype)1, c, rs_c, cs_c, &pr);                          \
  }                                                                                      \
  /* frame/l3/trmm.c:30-285: in place, from the original B */                            \
  int oracle_##s##trmm(mublis_side_t side, mublis_uplo_t uplo, mublis_trans_t ta,        \
                       mublis_diag_t diag, int m, int n, ctype alpha, const ctype *a,    \
                       int rs_a, int cs_a, ctype *b, int rs_b, int cs_b) {               \
    if (m == 0 || n == 0) return 0;                                                      \
    if (ta == MUBLIS_TRANSPOSE) { int t = rs_a; rs_a = cs_a; cs_a = t; uplo = flip_uplo(uplo); } \
    if (alpha == (ctype)0) {                                                             \
      for (long j = 0; j < n; ++j)                                                       \
        for (long i = 0; i < m; ++i) b[i * rs_b + j * cs_b] = 0;                         \
      return 0;                                                                          \
    }                                                                                    \
    mublis_l3_operand_t tri = {MUBLIS_STRUC_TRIANGULAR, uplo,                            \
                               diag == MUBLIS_UNIT_DIAG ? MUBLIS_PACKM_DIAG_UNIT         \
                                                        : MUBLIS_PACKM_DIAG_NONUNIT};    \
    ctype *src = (ctype *)malloc(sizeof(ctype) * (size_t)m * (size_t)n);                 \
    for (long j = 0; j < n; ++j)                                                         \
      for (long i = 0; i < m; ++i) src[i + j * (long)m] = b[i * rs_b + j * cs_b];        \
    mublis_l3_product_t pr = {{MUBLIS_L3_ALL, MUBLIS_L3_ALL, MUBLIS_L3_ALL},             \
                              side == MUBLIS_LEFT ? tri : OP_GENERAL,                    \
                              side == MUBLIS_RIGHT ? tri : OP_GENERAL};                  \
    int st;                                                                              \
    if (side == MUBLIS_LEFT)                                                             \
      st = oracle_l3_##s##driver(m, n, m, alpha, a, rs_a, cs_a, src, 1, m, (ctype)0, b,  \
                                 rs_b, cs_b, &pr);                                       \
    else                                                                                 \
      st = oracle_l3_##s##driver(m, n, n, alpha, src, 1, m, a, rs_a, cs_a, (ctype)0, b,  \
                                 rs_b, cs_b, &pr);                                       \
    free(src);                                                                           \
    return st;                                                                           \
  }                                                                                      \
  /* frame/l3/trsm.c:14-446: solve op(A) X = alpha B (left) / X op(A) = alpha B */       \
  int oracle_##s##trsm(mublis_side_t side, mublis_uplo_t uplo, mublis_trans_t ta,        \
                       mublis_diag_t diag, int m, int n, ctype alpha, const ctype *a,    \
                       int rs_a, int cs_a, ctype *b, int rs_b, int cs_b) {               \
    if (m == 0 || n == 0) return 0;                                                      \
    if (alpha == (ctype)0) {                                                             \
      for (long j = 0; j < n; ++j)                                                       \
        for (long i = 0; i < m; ++i) b[i * rs_b + j * cs_b] = 0;                         \
      return 0;                                                                          \
    }                                                                                    \
    if (side == MUBLIS_RIGHT) {                                                          \
      int t = m; m = n; n = t;                                                           \
      t = rs_b; rs_b = cs_b; cs_b = t;                                                   \
      ta = ta == MUBLIS_NO_TRANSPOSE ? MUBLIS_TRANSPOSE : MUBLIS_NO_TRANSPOSE;           \
    }                                                                                    \
    if (ta == MUBLIS_TRANSPOSE) { int t = rs_a; rs_a = cs_a; cs_a = t; uplo = flip_uplo(uplo); } \
    acc_t *x = (acc_t *)malloc(sizeof(acc_t) * (size_t)m);                               \
    for (long j = 0; j < n; ++j) {                                                       \
      for (long q = 0; q < m; ++q) {                                                     \
        long i = uplo == MUBLIS_LOWER ? q : m - 1 - q;                                   \
        acc_t r = (acc_t)alpha * (acc_t)b[i * rs_b + j * cs_b];                          \
        if (uplo == MUBLIS_LOWER)                                                        \
          for (long p = 0; p < i; ++p) r -= (acc_t)a[i * rs_a + p * cs_a] * x[p];        \
        else                                                                             \
          for (long p = i + 1; p < m; ++p) r -= (acc_t)a[i * rs_a + p * cs_a] * x[p];    \
        if (diag == MUBLIS_NON_UNIT_DIAG) r *= (acc_t)((ctype)1 / a[i * rs_a + i * cs_a]); \
        x[i] = r;                                                                        \
      }                                                                                  \
      for (long i = 0; i < m; ++i) b[i * rs_b + j * cs_b] = (ctype)x[i];                 \
    }                                                                                    \
    free(x);                                                                             \
    return 0;                                                                            \
  }
DEFINE_SHIMS(float, s)
DEFINE_SHIMS(double, d)

/* ---- seeded fills (column-major, leading dimension ld) ------------------ */

void oracle_fill_s(float *x, long m, long n, long ld, uint32_t seed, uint32_t id, int kind) {
  for (long j = 0; j < n; ++j)
    for (long i = 0; i < m; ++i)
      x[i + j * ld] = philox_draw_f32((uint64_t)(i + j * m), seed, id, kind);
}
void oracle_fill_d(double *x, long m, long n, long ld, uint32_t seed, uint32_t id, int kind) {
  for (long j = 0; j < n; ++j)
    for (long i = 0; i < m; ++i)
      x[i + j * ld] = philox_draw_f64((uint64_t)(i + j * m), seed, id, kind);
}
void oracle_philox(uint64_t index, uint32_t seed, uint32_t id, uint32_t out[4]) {
  philox4x32_t r = philox4x32_10(index, seed, id);
  memcpy(out, r.v, sizeof(r.v));
}
void oracle_philox_ctr(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  philox4x32_t r = philox4x32_10_ctr(ctr, key);
  memcpy(out, r.v, sizeof(r.v));
}

/* ---- double-double GEMM entries (error studies) ------------------------- */

static inline void two_sum(double a, double b, double *s, double *e) {
  double x = a + b, z = x - a;
  *s = x;
  *e = (a - (x - z)) + (b - z);
}

/* Entries (rows[q], cols[q]) of alpha*op(A)*op(B) + beta*C0, each returned as
 * an unevaluated sum hi[q] + lo[q] (Dot2, Ogita-Rump-Oishi 2005: error about
 * u^2 * cond + u).  A, B, C0 column-major; element types given by `is_f32`. */
void oracle_dd_gemm_entries(int is_f32, int ta, int tb, long k, double alpha, const void *a,
                            long lda, const void *b, long ldb, double beta, const void *c0,
                            long ldc, long count, const long *rows, const long *cols,
                            double *hi, double *lo) {
  /* Four entries at a time: their compensated sums are independent chains,
   * so interleaving them hides the latency of each chain's two_sum. */
  for (long q0 = 0; q0 < count; q0 += 4) {
    const int nq = count - q0 < 4 ? (int)(count - q0) : 4;
    double s4[4] = {0, 0, 0, 0}, e4[4] = {0, 0, 0, 0};
    long ia0[4], ias[4], ib0[4], ibs[4];
    for (int u = 0; u < 4; ++u) {
      long i = rows[q0 + (u < nq ? u : 0)], j = cols[q0 + (u < nq ? u : 0)];
      ia0[u] = ta ? i * lda : i;
      ias[u] = ta ? 1 : lda;
      ib0[u] = tb ? j : j * ldb;
      ibs[u] = tb ? ldb : 1;
    }
    for (long p = 0; p < k; ++p) {
      for (int u = 0; u < 4; ++u) {
        long ia = ia0[u] + p * ias[u], ib = ib0[u] + p * ibs[u];
        double x = is_f32 ? (double)((const float *)a)[ia] : ((const double *)a)[ia];
        double y = is_f32 ? (double)((const float *)b)[ib] : ((const double *)b)[ib];
        double ph = x * y, pl = fma(x, y, -ph);
        double t, te;
        two_sum(s4[u], ph, &t, &te);
        s4[u] = t;
        e4[u] += te + pl;
      }
    }
    for (int u = 0; u < nq; ++u) {
    const long q = q0 + u, i = rows[q], j = cols[q];
    const double s = s4[u], e = e4[u];
    /* alpha * (s + e) + beta * c, still compensated */
    double ah = alpha * s, al = fma(alpha, s, -ah) + alpha * e;
    double rh = ah, rl = al;
    if (beta != 0 && c0) {
      double cv = is_f32 ? (double)((const float *)c0)[i + j * ldc] : ((const double *)c0)[i + j * ldc];
      double bh = beta * cv, bl = fma(beta, cv, -bh);
      double t, te;
      two_sum(rh, bh, &t, &te);
      rh = t;
      rl += te + bl;
    }
    double t, te;
    two_sum(rh, rl, &t, &te);
    hi[q] = t;
    lo[q] = te;
    }
  }
}
