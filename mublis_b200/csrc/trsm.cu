// trsm.cu -- left triangular solve op(A) X = alpha B on the device.
//
// The reference (frame/l3/trsm.c) walks the diagonal in kc-blocks: pack the
// diagonal block with its diagonal inverted (:106-112, packm.c:143-144),
// solve it with gemmtrsm{l,u}_ukr (:139-158) and update the rows below with
// gemm_ukr (:166-274), all strictly in order along pc.  On the B200 the
// sequential part is kept small and the rest becomes large GEMMs:
//   * recursive halving: solve the top half, update the bottom half with one
//     GEMM (k = half the order, so it runs at GEMM speed), solve the bottom
//     half (upper: mirror image);
//   * leaves of at most 32 rows are solved by trsm_leaf_kernel: the leaf
//     triangle sits in shared memory with the reciprocal diagonal (computed
//     once, multiplied -- never divided -- as the reference does), each
//     thread owns one right-hand-side column in registers;
//   * the unit diagonal and the unstored triangle are never read.
// alpha is applied once up front (the reference's alpha_eff on the first
// block, trsm.c:96-97).
#include <cstring>

#include "kernels.cuh"

namespace {

constexpr int LEAF = 32;

template <typename T, int NB>
__global__ void __launch_bounds__(128) trsm_leaf_kernel(int mb, int n, const T *a, long rs_a,
                                                        long cs_a, T *b, long rs_b, long cs_b,
                                                        bool lower, bool unit) {
  __shared__ T L[NB][NB + 1];
  for (int idx = threadIdx.x; idx < NB * NB; idx += blockDim.x) {
    int i = idx % NB, p = idx / NB;
    T v = T(0);
    if (i < mb && p < mb) {
      if (i == p) v = unit ? T(1) : T(1) / a[i * rs_a + i * cs_a];
      else if (lower ? p < i : p > i) v = a[i * rs_a + p * cs_a];
    }
    L[i][p] = v;
  }
  __syncthreads();
  const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  T x[NB];
#pragma unroll
  for (int i = 0; i < NB; ++i) x[i] = i < mb ? b[i * rs_b + j * cs_b] : T(0);
  if (lower) {
#pragma unroll
    for (int i = 0; i < NB; ++i) {
      T r = x[i];
#pragma unroll
      for (int p = 0; p < i; ++p) r = fma(-L[i][p], x[p], r);
      x[i] = r * L[i][i];
    }
  } else {
#pragma unroll
    for (int i = NB - 1; i >= 0; --i) {
      T r = x[i];
#pragma unroll
      for (int p = i + 1; p < NB; ++p) r = fma(-L[i][p], x[p], r);
      x[i] = r * L[i][i];
    }
  }
#pragma unroll
  for (int i = 0; i < NB; ++i)
    if (i < mb) b[i * rs_b + j * cs_b] = x[i];
}

}  // namespace

template <typename T>
int launch_trsm_leaf(int mb, int n, const T *a, long rs_a, long cs_a, T *b, long rs_b, long cs_b,
                     bool lower, bool unit, cudaStream_t s) {
  if (mb <= 0 || n <= 0) return B200_OK;
  if (mb > LEAF) return b200_set_error(B200_EINVAL, "trsm leaf larger than 32");
  B200ProfScope prof(sizeof(T) == 4 ? "trsm_leaf_s" : "trsm_leaf_d", s);
  trsm_leaf_kernel<T, LEAF><<<(unsigned)b200_ceil_div(n, 128), 128, 0, s>>>(
      mb, n, a, rs_a, cs_a, b, rs_b, cs_b, lower, unit);
  B200_LAUNCH_CHECK();
  return B200_OK;
}

template int launch_trsm_leaf<float>(int, int, const float *, long, long, float *, long, long,
                                     bool, bool, cudaStream_t);
template int launch_trsm_leaf<double>(int, int, const double *, long, long, double *, long, long,
                                      bool, bool, cudaStream_t);

namespace {

template <typename T>
int trsm_rec(const b200_trsm_desc_t *d, long r0, long r1) {
  const T *a = (const T *)d->a;
  T *b = (T *)d->b;
  const bool lower = d->uplo == MUBLIS_LOWER;
  long rows = r1 - r0;
  if (rows <= LEAF)
    return launch_trsm_leaf<T>((int)rows, d->n, a + r0 * d->rs_a + r0 * d->cs_a, d->rs_a,
                               d->cs_a, b + r0 * d->rs_b, d->rs_b, d->cs_b, lower,
                               d->unit_diag != 0, b200_cur_stream());
  long half = b200_round_up((rows + 1) / 2, LEAF);
  long mid = r0 + half;
  // Rows solved first (src) and rows updated by them (dst).
  long s0 = lower ? r0 : mid, s1 = lower ? mid : r1;
  long t0 = lower ? mid : r0, t1 = lower ? r1 : mid;
  B200_TRY(trsm_rec<T>(d, s0, s1));
  b200_l3_desc_t g;
  memset(&g, 0, sizeof g);
  g.dtype = d->dtype;
  g.m = (int)(t1 - t0);
  g.n = d->n;
  g.k = (int)(s1 - s0);
  g.alpha = -1.0;
  g.beta = 1.0;
  g.npairs = 1;
  g.a[0] = a + t0 * d->rs_a + s0 * d->cs_a;
  g.rs_a[0] = d->rs_a;
  g.cs_a[0] = d->cs_a;
  g.b[0] = b + s0 * d->rs_b;
  g.rs_b[0] = d->rs_b;
  g.cs_b[0] = d->cs_b;
  g.c = b + t0 * d->rs_b;
  g.rs_c = d->rs_b;
  g.cs_c = d->cs_b;
  mublis_l3_operand_t gen = {MUBLIS_STRUC_GENERAL, MUBLIS_DENSE, MUBLIS_PACKM_DIAG_NONUNIT};
  g.product.domain.jp = g.product.domain.ji = g.product.domain.pi = MUBLIS_L3_ALL;
  g.product.a = gen;
  g.product.b = gen;
  g.form = d->form;
  g.slices = d->slices;
  B200_TRY(b200_l3_run(&g));
  return trsm_rec<T>(d, t0, t1);
}

}  // namespace

extern "C" int b200_trsm_run(const b200_trsm_desc_t *d) {
  if (d->m <= 0 || d->n <= 0) return B200_OK;
  if (d->uplo != MUBLIS_LOWER && d->uplo != MUBLIS_UPPER)
    return b200_set_error(B200_EINVAL, "trsm: uplo must be lower or upper");
  if (d->alpha != 1.0)
    B200_TRY(b200_scale_strided(d->dtype, d->m, d->n, d->alpha, d->b, d->rs_b, d->cs_b,
                                MUBLIS_L3_ALL));
  if (d->dtype == B200_F32) return trsm_rec<float>(d, 0, d->m);
  return trsm_rec<double>(d, 0, d->m);
}
