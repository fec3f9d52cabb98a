/*
 * context.c -- the "b200" target and config of the MuBLIS registry.
 *
 *   b200_context          a target context (include/mublis_instantiate.h:
 *                         125-155) whose micro-kernels run on the GPU
 *                         (ukr.cu); registered in include/target_registry.h
 *                         like the reference's targets/target_registry.h:6-12
 *   mublis_get_context    the config's dispatch (reference:
 *                         config/linux_avx2/dispatch.c:4-8), returning
 *                         b200_context when an sm_100 device is usable
 *   mublis_get_safe_context
 *                         once-only validated copy, as the reference's
 *                         frame/base/safe_dispatch.c:10-71 (pthread_once,
 *                         non-null kernels, positive sizes, mc % mr,
 *                         nc % nr, kc % mr, kc % nr)
 *
 * Block sizes describe the device tiling: mr x nr is the micro-tile the
 * context's kernels compute (32 x 32), mc / nc the CTA tile of the plain
 * kernels and kc a multiple of both.
 */
#include <pthread.h>
#include <stddef.h>

#include "../../../include/mublis_instantiate.h"
#include "../../../include/target_registry.h"
#include "../b200_internal.h"

#define B200_MR 32
#define B200_NR 32

static void b200_sgemm_ukr(int k, float alpha, const float *restrict a, const float *restrict b,
                           float beta, float *restrict c, int rs_c, int cs_c,
                           const mublis_auxinfo_t *aux) {
  (void)aux;
  b200_ukr_gemm(B200_F32, k, &alpha, a, b, &beta, c, rs_c, cs_c, B200_MR, B200_NR);
}
static void b200_dgemm_ukr(int k, double alpha, const double *restrict a,
                           const double *restrict b, double beta, double *restrict c, int rs_c,
                           int cs_c, const mublis_auxinfo_t *aux) {
  (void)aux;
  b200_ukr_gemm(B200_F64, k, &alpha, a, b, &beta, c, rs_c, cs_c, B200_MR, B200_NR);
}

#define STAMP_TRSM_UKR(ctype, name, DT, LOWER)                                               \
  static void name(int k, ctype alpha, const ctype *restrict a1x, const ctype *restrict a11, \
                   const ctype *restrict bx1, ctype *restrict b11, ctype *restrict c11,      \
                   int rs_c, int cs_c, const mublis_auxinfo_t *aux) {                        \
    (void)aux;                                                                               \
    b200_ukr_gemmtrsm(DT, LOWER, k, &alpha, a1x, a11, bx1, b11, c11, rs_c, cs_c, B200_MR,    \
                      B200_NR);                                                              \
  }
STAMP_TRSM_UKR(float, b200_sgemmtrsml_ukr, B200_F32, 1)
STAMP_TRSM_UKR(float, b200_sgemmtrsmu_ukr, B200_F32, 0)
STAMP_TRSM_UKR(double, b200_dgemmtrsml_ukr, B200_F64, 1)
STAMP_TRSM_UKR(double, b200_dgemmtrsmu_ukr, B200_F64, 0)

MUBLIS_CONTEXT_STAMP(b200_context,
                     b200_sgemm_ukr, b200_sgemmtrsml_ukr, b200_sgemmtrsmu_ukr,
                     B200_MR, B200_NR, 128, 128, 128,
                     b200_dgemm_ukr, b200_dgemmtrsml_ukr, b200_dgemmtrsmu_ukr,
                     B200_MR, B200_NR, 128, 128, 64)

/* config/b200: select b200_context once a usable device is present. */
int mublis_get_context(mublis_context_t *context) {
  if (context == NULL) return 1;
  int st = b200_init();
  if (st != 0) return st;
  *context = b200_context;
  return 0;
}

static pthread_once_t g_once = PTHREAD_ONCE_INIT;
static mublis_context_t g_ctx;
static int g_ctx_status = 1;

static int valid(int mr, int nr, int mc, int kc, int nc, const void *g, const void *l,
                 const void *u) {
  return g && l && u && mr > 0 && nr > 0 && mc > 0 && kc > 0 && nc > 0 && mc % mr == 0 &&
         nc % nr == 0 && kc % mr == 0 && kc % nr == 0;
}

static void init_ctx(void) {
  mublis_context_t c = {0};
  g_ctx_status = mublis_get_context(&c);
  if (g_ctx_status != 0) return;
  if (!valid(c.s.mr, c.s.nr, c.s.mc, c.s.kc, c.s.nc, (const void *)c.s.gemm_ukr,
             (const void *)c.s.gemmtrsml_ukr, (const void *)c.s.gemmtrsmu_ukr) ||
      !valid(c.d.mr, c.d.nr, c.d.mc, c.d.kc, c.d.nc, (const void *)c.d.gemm_ukr,
             (const void *)c.d.gemmtrsml_ukr, (const void *)c.d.gemmtrsmu_ukr)) {
    g_ctx_status = 1;
    return;
  }
  g_ctx = c;
}

int mublis_get_safe_context(const mublis_context_t **context) {
  if (context == NULL) return 1;
  pthread_once(&g_once, init_ctx);
  *context = g_ctx_status == 0 ? &g_ctx : NULL;
  return g_ctx_status;
}
