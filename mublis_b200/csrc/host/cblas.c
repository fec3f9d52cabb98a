/*
 * cblas.c -- CBLAS Level-3 layer of the B200 build.
 *
 * Same observable behaviour as the reference's frame/compat/cblas/cblas.c:
 *   - weak cblas_xerbla that prints to stderr and exits (:14-32);
 *   - netlib-style argument checks with the netlib parameter positions
 *     (CBLAS_CHECK :92-98 and each routine's checks);
 *   - a nonzero backend status is reported through cblas_xerbla(0, ...)
 *     (:100-112);
 *   - column-major calls pass (rs, cs) = (1, ld) (:179-182); row-major calls
 *     are re-expressed column-major: GEMM as C^T = op(B)^T op(A)^T with A/B
 *     and M/N swapped (:188-200); SYMM/TRMM/TRSM flip side and uplo and swap
 *     M/N (:266-277, :503-515); SYRK/SYR2K flip uplo and trans
 *     (:341-351, :421-432).
 */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>

#include "../../../include/cblas.h"
#include "../../../include/mublis.h"
#include "../../../include/mublis_b200.h"

__attribute__((weak)) void cblas_xerbla(int p, const char *rout, const char *form, ...) {
  va_list args;
  if (p > 0)
    fprintf(stderr, "Parameter %d to routine %s was incorrect\n", p, rout);
  else
    fprintf(stderr, "Routine %s failed\n", rout);
  va_start(args, form);
  vfprintf(stderr, form, args);
  va_end(args);
  exit(EXIT_FAILURE);
}

static int at_least1(int v) { return v > 1 ? v : 1; }
static int ok_order(int v) { return v == CblasRowMajor || v == CblasColMajor; }
static int ok_trans(int v) { return v == CblasNoTrans || v == CblasTrans; }
static int ok_uplo(int v) { return v == CblasUpper || v == CblasLower; }
static int ok_diag(int v) { return v == CblasNonUnit || v == CblasUnit; }
static int ok_side(int v) { return v == CblasLeft || v == CblasRight; }

static mublis_trans_t tr(int v) { return v == CblasNoTrans ? MUBLIS_NO_TRANSPOSE : MUBLIS_TRANSPOSE; }
static mublis_trans_t tr_flip(int v) {
  return v == CblasNoTrans ? MUBLIS_TRANSPOSE : MUBLIS_NO_TRANSPOSE;
}
static mublis_uplo_t up(int v) { return v == CblasUpper ? MUBLIS_UPPER : MUBLIS_LOWER; }
static mublis_uplo_t up_flip(int v) { return v == CblasUpper ? MUBLIS_LOWER : MUBLIS_UPPER; }
static mublis_diag_t dg(int v) { return v == CblasUnit ? MUBLIS_UNIT_DIAG : MUBLIS_NON_UNIT_DIAG; }
static mublis_side_t sd(int v) { return v == CblasLeft ? MUBLIS_LEFT : MUBLIS_RIGHT; }
static mublis_side_t sd_flip(int v) { return v == CblasLeft ? MUBLIS_RIGHT : MUBLIS_LEFT; }

#define REQUIRE(cond, pos, rout, ...)          \
  do {                                         \
    if (!(cond)) {                             \
      cblas_xerbla((pos), (rout), __VA_ARGS__); \
      return;                                  \
    }                                          \
  } while (0)

static void finish(int status, const char *rout) {
  if (status != 0)
    cblas_xerbla(0, rout, "MuBLIS backend returned status %d (%s)\n", status,
                 mublis_b200_last_error());
}

#define STAMP_GEMM(p, T)                                                                     \
  void cblas_##p##gemm(const enum CBLAS_ORDER Order, const enum CBLAS_TRANSPOSE TransA,      \
                       const enum CBLAS_TRANSPOSE TransB, const int M, const int N,          \
                       const int K, const T alpha, const T *A, const int lda, const T *B,    \
                       const int ldb, const T beta, T *C, const int ldc) {                   \
    const char *r = "cblas_" #p "gemm";                                                      \
    REQUIRE(ok_order(Order), 1, r, "Illegal Order setting, %d\n", Order);                    \
    REQUIRE(ok_trans(TransA), 2, r, "Illegal TransA setting, %d\n", TransA);                 \
    REQUIRE(ok_trans(TransB), 3, r, "Illegal TransB setting, %d\n", TransB);                 \
    REQUIRE(M >= 0, 4, r, "M must be nonnegative, %d\n", M);                                 \
    REQUIRE(N >= 0, 5, r, "N must be nonnegative, %d\n", N);                                 \
    REQUIRE(K >= 0, 6, r, "K must be nonnegative, %d\n", K);                                 \
    int col = Order == CblasColMajor;                                                        \
    int min_lda = at_least1(col ? (TransA == CblasNoTrans ? M : K)                           \
                                : (TransA == CblasNoTrans ? K : M));                         \
    int min_ldb = at_least1(col ? (TransB == CblasNoTrans ? K : N)                           \
                                : (TransB == CblasNoTrans ? N : K));                         \
    REQUIRE(lda >= min_lda, 9, r, "lda must be at least %d, %d\n", min_lda, lda);            \
    REQUIRE(ldb >= min_ldb, 11, r, "ldb must be at least %d, %d\n", min_ldb, ldb);           \
    REQUIRE(ldc >= at_least1(col ? M : N), 14, r, "ldc is too small, %d\n", ldc);            \
    if (col)                                                                                 \
      finish(mublis_##p##gemm(tr(TransA), tr(TransB), M, N, K, alpha, A, 1, lda, B, 1, ldb,  \
                              beta, C, 1, ldc), r);                                          \
    else                                                                                     \
      finish(mublis_##p##gemm(tr(TransB), tr(TransA), N, M, K, alpha, B, 1, ldb, A, 1, lda,  \
                              beta, C, 1, ldc), r);                                          \
  }

#define STAMP_SYMM(p, T)                                                                     \
  void cblas_##p##symm(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,             \
                       const enum CBLAS_UPLO Uplo, const int M, const int N, const T alpha,  \
                       const T *A, const int lda, const T *B, const int ldb, const T beta,   \
                       T *C, const int ldc) {                                                \
    const char *r = "cblas_" #p "symm";                                                      \
    REQUIRE(ok_order(Order), 1, r, "Illegal Order setting, %d\n", Order);                    \
    REQUIRE(ok_side(Side), 2, r, "Illegal Side setting, %d\n", Side);                        \
    REQUIRE(ok_uplo(Uplo), 3, r, "Illegal Uplo setting, %d\n", Uplo);                        \
    REQUIRE(M >= 0, 4, r, "M must be nonnegative, %d\n", M);                                 \
    REQUIRE(N >= 0, 5, r, "N must be nonnegative, %d\n", N);                                 \
    REQUIRE(lda >= at_least1(Side == CblasLeft ? M : N), 8, r, "lda is too small, %d\n",     \
            lda);                                                                            \
    int col = Order == CblasColMajor;                                                        \
    int min_bc = at_least1(col ? M : N);                                                     \
    REQUIRE(ldb >= min_bc, 10, r, "ldb must be at least %d, %d\n", min_bc, ldb);             \
    REQUIRE(ldc >= min_bc, 13, r, "ldc must be at least %d, %d\n", min_bc, ldc);             \
    if (col)                                                                                 \
      finish(mublis_##p##symm(sd(Side), up(Uplo), M, N, alpha, A, 1, lda, B, 1, ldb, beta,   \
                              C, 1, ldc), r);                                                \
    else                                                                                     \
      finish(mublis_##p##symm(sd_flip(Side), up_flip(Uplo), N, M, alpha, A, 1, lda, B, 1,    \
                              ldb, beta, C, 1, ldc), r);                                     \
  }

#define STAMP_SYRK(p, T)                                                                     \
  void cblas_##p##syrk(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,             \
                       const enum CBLAS_TRANSPOSE Trans, const int N, const int K,           \
                       const T alpha, const T *A, const int lda, const T beta, T *C,         \
                       const int ldc) {                                                      \
    const char *r = "cblas_" #p "syrk";                                                      \
    REQUIRE(ok_order(Order), 1, r, "Illegal Order setting, %d\n", Order);                    \
    REQUIRE(ok_uplo(Uplo), 2, r, "Illegal Uplo setting, %d\n", Uplo);                        \
    REQUIRE(ok_trans(Trans), 3, r, "Illegal Trans setting, %d\n", Trans);                    \
    REQUIRE(N >= 0, 4, r, "N must be nonnegative, %d\n", N);                                 \
    REQUIRE(K >= 0, 5, r, "K must be nonnegative, %d\n", K);                                 \
    int col = Order == CblasColMajor;                                                        \
    int min_lda = at_least1(col ? (Trans == CblasNoTrans ? N : K)                            \
                                : (Trans == CblasNoTrans ? K : N));                          \
    REQUIRE(lda >= min_lda, 8, r, "lda must be at least %d, %d\n", min_lda, lda);            \
    REQUIRE(ldc >= at_least1(N), 11, r, "ldc is too small, %d\n", ldc);                      \
    if (col)                                                                                 \
      finish(mublis_##p##syrk(up(Uplo), tr(Trans), N, K, alpha, A, 1, lda, beta, C, 1, ldc), \
             r);                                                                             \
    else                                                                                     \
      finish(mublis_##p##syrk(up_flip(Uplo), tr_flip(Trans), N, K, alpha, A, 1, lda, beta,  \
                              C, 1, ldc), r);                                                \
  }

#define STAMP_SYR2K(p, T)                                                                    \
  void cblas_##p##syr2k(const enum CBLAS_ORDER Order, const enum CBLAS_UPLO Uplo,            \
                        const enum CBLAS_TRANSPOSE Trans, const int N, const int K,          \
                        const T alpha, const T *A, const int lda, const T *B, const int ldb, \
                        const T beta, T *C, const int ldc) {                                 \
    const char *r = "cblas_" #p "syr2k";                                                     \
    REQUIRE(ok_order(Order), 1, r, "Illegal Order setting, %d\n", Order);                    \
    REQUIRE(ok_uplo(Uplo), 2, r, "Illegal Uplo setting, %d\n", Uplo);                        \
    REQUIRE(ok_trans(Trans), 3, r, "Illegal Trans setting, %d\n", Trans);                    \
    REQUIRE(N >= 0, 4, r, "N must be nonnegative, %d\n", N);                                 \
    REQUIRE(K >= 0, 5, r, "K must be nonnegative, %d\n", K);                                 \
    int col = Order == CblasColMajor;                                                        \
    int min_ab = at_least1(col ? (Trans == CblasNoTrans ? N : K)                             \
                               : (Trans == CblasNoTrans ? K : N));                           \
    REQUIRE(lda >= min_ab, 8, r, "lda must be at least %d, %d\n", min_ab, lda);              \
    REQUIRE(ldb >= min_ab, 10, r, "ldb must be at least %d, %d\n", min_ab, ldb);             \
    REQUIRE(ldc >= at_least1(N), 13, r, "ldc is too small, %d\n", ldc);                      \
    if (col)                                                                                 \
      finish(mublis_##p##syr2k(up(Uplo), tr(Trans), N, K, alpha, A, 1, lda, B, 1, ldb, beta, \
                               C, 1, ldc), r);                                               \
    else                                                                                     \
      finish(mublis_##p##syr2k(up_flip(Uplo), tr_flip(Trans), N, K, alpha, A, 1, lda, B, 1,  \
                               ldb, beta, C, 1, ldc), r);                                    \
  }

#define STAMP_TR(p, name, T)                                                                 \
  void cblas_##p##name(const enum CBLAS_ORDER Order, const enum CBLAS_SIDE Side,             \
                       const enum CBLAS_UPLO Uplo, const enum CBLAS_TRANSPOSE TransA,        \
                       const enum CBLAS_DIAG Diag, const int M, const int N, const T alpha,  \
                       const T *A, const int lda, T *B, const int ldb) {                     \
    const char *r = "cblas_" #p #name;                                                       \
    REQUIRE(ok_order(Order), 1, r, "Illegal Order setting, %d\n", Order);                    \
    REQUIRE(ok_side(Side), 2, r, "Illegal Side setting, %d\n", Side);                        \
    REQUIRE(ok_uplo(Uplo), 3, r, "Illegal Uplo setting, %d\n", Uplo);                        \
    REQUIRE(ok_trans(TransA), 4, r, "Illegal TransA setting, %d\n", TransA);                 \
    REQUIRE(ok_diag(Diag), 5, r, "Illegal Diag setting, %d\n", Diag);                        \
    REQUIRE(M >= 0, 6, r, "M must be nonnegative, %d\n", M);                                 \
    REQUIRE(N >= 0, 7, r, "N must be nonnegative, %d\n", N);                                 \
    REQUIRE(lda >= at_least1(Side == CblasLeft ? M : N), 10, r, "lda is too small, %d\n",    \
            lda);                                                                            \
    int col = Order == CblasColMajor;                                                        \
    int min_ldb = at_least1(col ? M : N);                                                    \
    REQUIRE(ldb >= min_ldb, 12, r, "ldb must be at least %d, %d\n", min_ldb, ldb);           \
    if (col)                                                                                 \
      finish(mublis_##p##name(sd(Side), up(Uplo), tr(TransA), dg(Diag), M, N, alpha, A, 1,   \
                              lda, B, 1, ldb), r);                                           \
    else                                                                                     \
      finish(mublis_##p##name(sd_flip(Side), up_flip(Uplo), tr(TransA), dg(Diag), N, M,     \
                              alpha, A, 1, lda, B, 1, ldb), r);                              \
  }

STAMP_GEMM(s, float)
STAMP_GEMM(d, double)
STAMP_SYMM(s, float)
STAMP_SYMM(d, double)
STAMP_SYRK(s, float)
STAMP_SYRK(d, double)
STAMP_SYR2K(s, float)
STAMP_SYR2K(d, double)
STAMP_TR(s, trmm, float)
STAMP_TR(d, trmm, double)
STAMP_TR(s, trsm, float)
STAMP_TR(d, trsm, double)
