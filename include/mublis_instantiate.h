/*
 * mublis_instantiate.h -- target/config interface of MuBLIS, B200 build.
 *
 * Same ABI as the reference's include/mublis_instantiate.h:
 *   mublis_auxinfo_t                          :29-31
 *   GEMM micro-kernel pointer types           :53-70
 *   GEMMTRSM micro-kernel pointer types       :95-114
 *   mublis_{s,d}context_t, mublis_context_t   :125-155
 *   MUBLIS_CONTEXT_STAMP                      :202-236
 *   mublis_get_context                        :247
 *
 * Micro-kernel contract (unchanged):
 *   gemm_ukr:     C(MR x NR) := alpha * A * B + beta * C, A(i,p) = a[p*MR+i],
 *                 B(p,j) = b[p*NR+j], C(i,j) = c[i*rs_c + j*cs_c]; beta == 0
 *                 means C is not read.
 *   gemmtrsm_ukr: R := alpha * B11 - A1x * Bx1, then A11 X = R with A11 an
 *                 MR x MR column-major triangle whose diagonal is already
 *                 inverted; X overwrites the row-major MR x NR b11 and is
 *                 stored to c11.  k may be 0.
 *
 * In the B200 build (target "b200", registered in target_registry.h) the
 * micro-kernels run on the GPU: each call stages its packed panels to the
 * device, runs one MR x NR tile there, and copies the tile back.  They exist
 * for contract tests and for external code that drives its own loops; the
 * library's own routines never call them (they tile whole problems on the
 * device instead).
 */
#ifndef MUBLIS_INSTANTIATE_H
#define MUBLIS_INSTANTIATE_H

#ifdef __cplusplus
#define MUBLIS_RESTRICT __restrict__
extern "C" {
#else
#define MUBLIS_RESTRICT restrict
#endif

typedef struct {
  const void *c_next; /* optional prefetch hint: the tile visited next */
} mublis_auxinfo_t;

typedef void (*mublis_sgemm_ukr_ft)(int k, float alpha, const float *MUBLIS_RESTRICT a,
                                    const float *MUBLIS_RESTRICT b, float beta,
                                    float *MUBLIS_RESTRICT c, int rs_c, int cs_c,
                                    const mublis_auxinfo_t *aux);
typedef void (*mublis_dgemm_ukr_ft)(int k, double alpha, const double *MUBLIS_RESTRICT a,
                                    const double *MUBLIS_RESTRICT b, double beta,
                                    double *MUBLIS_RESTRICT c, int rs_c, int cs_c,
                                    const mublis_auxinfo_t *aux);

typedef void (*mublis_sgemmtrsml_ukr_ft)(int k, float alpha, const float *MUBLIS_RESTRICT a1x,
                                         const float *MUBLIS_RESTRICT a11,
                                         const float *MUBLIS_RESTRICT bx1,
                                         float *MUBLIS_RESTRICT b11, float *MUBLIS_RESTRICT c11,
                                         int rs_c, int cs_c, const mublis_auxinfo_t *aux);
typedef mublis_sgemmtrsml_ukr_ft mublis_sgemmtrsmu_ukr_ft;
typedef void (*mublis_dgemmtrsml_ukr_ft)(int k, double alpha, const double *MUBLIS_RESTRICT a1x,
                                         const double *MUBLIS_RESTRICT a11,
                                         const double *MUBLIS_RESTRICT bx1,
                                         double *MUBLIS_RESTRICT b11, double *MUBLIS_RESTRICT c11,
                                         int rs_c, int cs_c, const mublis_auxinfo_t *aux);
typedef mublis_dgemmtrsml_ukr_ft mublis_dgemmtrsmu_ukr_ft;

/* Kernels and block sizes of one precision.  All sizes positive; mc % mr,
 * nc % nr, kc % mr and kc % nr must be 0. */
typedef struct {
  mublis_sgemm_ukr_ft gemm_ukr;
  mublis_sgemmtrsml_ukr_ft gemmtrsml_ukr;
  mublis_sgemmtrsmu_ukr_ft gemmtrsmu_ukr;
  int mr, nr;
  int mc, kc, nc;
} mublis_scontext_t;

typedef struct {
  mublis_dgemm_ukr_ft gemm_ukr;
  mublis_dgemmtrsml_ukr_ft gemmtrsml_ukr;
  mublis_dgemmtrsmu_ukr_ft gemmtrsmu_ukr;
  int mr, nr;
  int mc, kc, nc;
} mublis_dcontext_t;

typedef struct {
  mublis_scontext_t s;
  mublis_dcontext_t d;
} mublis_context_t;

#define MUBLIS_GEMM_UKR_PROT_STAMP(ctype, name)                                          \
  void name(int k, ctype alpha, const ctype *MUBLIS_RESTRICT a,                          \
            const ctype *MUBLIS_RESTRICT b, ctype beta, ctype *MUBLIS_RESTRICT c,        \
            int rs_c, int cs_c, const mublis_auxinfo_t *aux);

#define MUBLIS_GEMMTRSM_UKR_PROT_STAMP(ctype, name)                                      \
  void name(int k, ctype alpha, const ctype *MUBLIS_RESTRICT a1x,                        \
            const ctype *MUBLIS_RESTRICT a11, const ctype *MUBLIS_RESTRICT bx1,          \
            ctype *MUBLIS_RESTRICT b11, ctype *MUBLIS_RESTRICT c11, int rs_c, int cs_c,  \
            const mublis_auxinfo_t *aux);

/* Defines `const mublis_context_t context_name` from the single-precision
 * group (3 kernels, mr, nr, mc, kc, nc) and the double-precision group. */
#define MUBLIS_CONTEXT_STAMP(context_name, s_gemm, s_trsml, s_trsmu, s_mr, s_nr, s_mc,    \
                             s_kc, s_nc, d_gemm, d_trsml, d_trsmu, d_mr, d_nr, d_mc,     \
                             d_kc, d_nc)                                                 \
  const mublis_context_t context_name = {                                                \
      {(s_gemm), (s_trsml), (s_trsmu), (s_mr), (s_nr), (s_mc), (s_kc), (s_nc)},          \
      {(d_gemm), (d_trsml), (d_trsmu), (d_mr), (d_nr), (d_mc), (d_kc), (d_nc)}};

/* Selects the target context; 0 on success.  The b200 config returns
 * b200_context once a usable sm_100 device is present, nonzero otherwise. */
int mublis_get_context(mublis_context_t *context);

#ifdef __cplusplus
}
#endif

#endif
