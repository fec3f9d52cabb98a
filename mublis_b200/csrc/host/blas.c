/*
 * blas.c -- the twelve MuBLIS BLAS mirrors (include/mublis.h:85-197).
 *
 * Each builds the same product descriptor as the reference shim and hands
 * it to the device driver:
 *   GEMM   frame/l3/gemm.c:14-52   op() becomes a stride swap, domain ALL
 *   SYMM   frame/l3/symm.c:14-56   symmetric operand + uplo; a right-side
 *                                  SYMM swaps the roles of A and B
 *   SYRK   frame/l3/syrk.c:19-51   ji = uplo's relation, B = A with strides
 *                                  swapped
 *   SYR2K  frame/l3/syr2k.c:47-68  the reference makes two driver passes (the
 *                                  second with beta = 1); here both products
 *                                  are one descriptor with two (A, B) pairs
 *                                  concatenated along k, i.e. one pass
 *   TRMM / TRSM                    front.c
 */
#include <string.h>

#include "front.h"

static const mublis_l3_operand_t GEN = {MUBLIS_STRUC_GENERAL, MUBLIS_DENSE,
                                        MUBLIS_PACKM_DIAG_NONUNIT};

static void desc_init(b200_l3_desc_t *d, int dtype, int m, int n, int k, double alpha,
                      double beta, void *c, int rs_c, int cs_c) {
  memset(d, 0, sizeof *d);
  d->dtype = dtype;
  d->m = m;
  d->n = n;
  d->k = k;
  d->alpha = alpha;
  d->beta = beta;
  d->npairs = 1;
  d->c = c;
  d->rs_c = rs_c;
  d->cs_c = cs_c;
  d->product.domain.jp = d->product.domain.ji = d->product.domain.pi = MUBLIS_L3_ALL;
  d->product.a = GEN;
  d->product.b = GEN;
  d->form = B200_FORM_AUTO;
}

static void set_pair(b200_l3_desc_t *d, int t, const void *a, long rs_a, long cs_a,
                     const void *b, long rs_b, long cs_b) {
  d->a[t] = a; d->rs_a[t] = rs_a; d->cs_a[t] = cs_a;
  d->b[t] = b; d->rs_b[t] = rs_b; d->cs_b[t] = cs_b;
}

static mublis_l3_relation_t rel_of(mublis_uplo_t u) {
  return u == MUBLIS_LOWER ? MUBLIS_L3_LOWER : (u == MUBLIS_UPPER ? MUBLIS_L3_UPPER : MUBLIS_L3_ALL);
}

static int gemm(int dt, mublis_trans_t ta, mublis_trans_t tb, int m, int n, int k, double alpha,
                const void *a, int rs_a, int cs_a, const void *b, int rs_b, int cs_b, double beta,
                void *c, int rs_c, int cs_c) {
  if (ta == MUBLIS_TRANSPOSE) { int t = rs_a; rs_a = cs_a; cs_a = t; }
  if (tb == MUBLIS_TRANSPOSE) { int t = rs_b; rs_b = cs_b; cs_b = t; }
  b200_l3_desc_t d;
  desc_init(&d, dt, m, n, k, alpha, beta, c, rs_c, cs_c);
  set_pair(&d, 0, a, rs_a, cs_a, b, rs_b, cs_b);
  return b200_front_l3(&d);
}

static int symm(int dt, mublis_side_t side, mublis_uplo_t uplo, int m, int n, double alpha,
                const void *a, int rs_a, int cs_a, const void *b, int rs_b, int cs_b, double beta,
                void *c, int rs_c, int cs_c) {
  mublis_l3_operand_t sym = {MUBLIS_STRUC_SYMMETRIC, uplo, MUBLIS_PACKM_DIAG_NONUNIT};
  b200_l3_desc_t d;
  if (side == MUBLIS_LEFT) {
    desc_init(&d, dt, m, n, m, alpha, beta, c, rs_c, cs_c);
    d.product.a = sym;
    set_pair(&d, 0, a, rs_a, cs_a, b, rs_b, cs_b);
  } else {
    desc_init(&d, dt, m, n, n, alpha, beta, c, rs_c, cs_c);
    d.product.b = sym;
    set_pair(&d, 0, b, rs_b, cs_b, a, rs_a, cs_a);
  }
  return b200_front_l3(&d);
}

static int syrk(int dt, mublis_uplo_t uplo, mublis_trans_t trans, int n, int k, double alpha,
                const void *a, int rs_a, int cs_a, double beta, void *c, int rs_c, int cs_c) {
  if (trans == MUBLIS_TRANSPOSE) { int t = rs_a; rs_a = cs_a; cs_a = t; }
  b200_l3_desc_t d;
  desc_init(&d, dt, n, n, k, alpha, beta, c, rs_c, cs_c);
  d.product.domain.ji = rel_of(uplo);
  set_pair(&d, 0, a, rs_a, cs_a, a, cs_a, rs_a);
  return b200_front_l3(&d);
}

static int syr2k(int dt, mublis_uplo_t uplo, mublis_trans_t trans, int n, int k, double alpha,
                 const void *a, int rs_a, int cs_a, const void *b, int rs_b, int cs_b,
                 double beta, void *c, int rs_c, int cs_c) {
  if (trans == MUBLIS_TRANSPOSE) {
    int t = rs_a; rs_a = cs_a; cs_a = t;
    t = rs_b; rs_b = cs_b; cs_b = t;
  }
  b200_l3_desc_t d;
  desc_init(&d, dt, n, n, k, alpha, beta, c, rs_c, cs_c);
  d.product.domain.ji = rel_of(uplo);
  d.npairs = 2;
  set_pair(&d, 0, a, rs_a, cs_a, b, cs_b, rs_b); /* alpha A B^T */
  set_pair(&d, 1, b, rs_b, cs_b, a, cs_a, rs_a); /* alpha B A^T */
  return b200_front_l3(&d);
}

#define STAMP_MIRRORS(ctype, p, DT)                                                          \
  int mublis_##p##gemm(mublis_trans_t ta, mublis_trans_t tb, int m, int n, int k,            \
                       ctype alpha, const ctype *a, int rs_a, int cs_a, const ctype *b,      \
                       int rs_b, int cs_b, ctype beta, ctype *c, int rs_c, int cs_c) {       \
    return gemm(DT, ta, tb, m, n, k, alpha, a, rs_a, cs_a, b, rs_b, cs_b, beta, c, rs_c,     \
                cs_c);                                                                       \
  }                                                                                          \
  int mublis_##p##symm(mublis_side_t side, mublis_uplo_t uplo, int m, int n, ctype alpha,    \
                       const ctype *a, int rs_a, int cs_a, const ctype *b, int rs_b,         \
                       int cs_b, ctype beta, ctype *c, int rs_c, int cs_c) {                 \
    return symm(DT, side, uplo, m, n, alpha, a, rs_a, cs_a, b, rs_b, cs_b, beta, c, rs_c,    \
                cs_c);                                                                       \
  }                                                                                          \
  int mublis_##p##syrk(mublis_uplo_t uplo, mublis_trans_t trans, int n, int k, ctype alpha,  \
                       const ctype *a, int rs_a, int cs_a, ctype beta, ctype *c, int rs_c,   \
                       int cs_c) {                                                           \
    return syrk(DT, uplo, trans, n, k, alpha, a, rs_a, cs_a, beta, c, rs_c, cs_c);           \
  }                                                                                          \
  int mublis_##p##syr2k(mublis_uplo_t uplo, mublis_trans_t trans, int n, int k, ctype alpha, \
                        const ctype *a, int rs_a, int cs_a, const ctype *b, int rs_b,        \
                        int cs_b, ctype beta, ctype *c, int rs_c, int cs_c) {                \
    return syr2k(DT, uplo, trans, n, k, alpha, a, rs_a, cs_a, b, rs_b, cs_b, beta, c, rs_c,  \
                 cs_c);                                                                      \
  }                                                                                          \
  int mublis_##p##trmm(mublis_side_t side, mublis_uplo_t uplo, mublis_trans_t ta,            \
                       mublis_diag_t diag, int m, int n, ctype alpha, const ctype *a,        \
                       int rs_a, int cs_a, ctype *b, int rs_b, int cs_b) {                   \
    return b200_front_trmm(DT, side, uplo, ta, diag, m, n, alpha, a, rs_a, cs_a, b, rs_b,    \
                           cs_b);                                                            \
  }                                                                                          \
  int mublis_##p##trsm(mublis_side_t side, mublis_uplo_t uplo, mublis_trans_t ta,            \
                       mublis_diag_t diag, int m, int n, ctype alpha, const ctype *a,        \
                       int rs_a, int cs_a, ctype *b, int rs_b, int cs_b) {                   \
    return b200_front_trsm(DT, side, uplo, ta, diag, m, n, alpha, a, rs_a, cs_a, b, rs_b,    \
                           cs_b);                                                            \
  }

STAMP_MIRRORS(float, s, B200_F32)
STAMP_MIRRORS(double, d, B200_F64)
