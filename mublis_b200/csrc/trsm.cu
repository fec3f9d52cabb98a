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
//   * leaves are the 64 x 64 diagonal blocks.  All of them are inverted up
//     front in one launch (trsm_inv_diag_kernel: substitution against the
//     reciprocal diagonal, computed once and multiplied -- never divided --
//     as the reference does; the unstored triangle and a unit diagonal are
//     never read), so each leaf solve is X_b = inv(A_bb) B_b, a parallel
//     64 x n GEMM instead of a 64-deep dependent chain per column;
//   * updates and leaf products with k <= 256 read their operands directly
//     (no pack pass); larger ones use the packed driver path;
//   * the unit diagonal and the unstored triangle are never read.
// alpha is applied once up front (the reference's alpha_eff on the first
// block, trsm.c:96-97).
#include <cstring>

#include "kernels.cuh"

namespace {

constexpr int LEAF = 64;  // rows per diagonal block (leaf)

// One CTA per diagonal block: thread j computes column j of the inverse of
// the block's (lower or upper) triangle by substitution, L x = e_j.  Rows
// past the matrix order are padded with the identity.  Output: block b as a
// LEAF x LEAF column-major matrix at inv + b * LEAF * LEAF.
template <typename T>
__global__ void __launch_bounds__(LEAF) trsm_inv_diag_kernel(int m, const T *a, long rs_a,
                                                              long cs_a, bool lower, bool unit,
                                                              T *inv) {
  __shared__ T L[LEAF][LEAF + 1];
  const int b = blockIdx.x, j = threadIdx.x;
  const long r0 = (long)b * LEAF;
  const int mb = (int)min((long)LEAF, m - r0);
  const bool rows_fast = labs(rs_a) <= labs(cs_a);
  for (int idx = j; idx < LEAF * LEAF; idx += LEAF) {
    int i = rows_fast ? idx % LEAF : idx / LEAF, p = rows_fast ? idx / LEAF : idx % LEAF;
    T v = T(0);
    if (i < mb && p < mb) {
      if (i == p) v = unit ? T(1) : T(1) / a[(r0 + i) * rs_a + (r0 + i) * cs_a];
      else if (lower ? p < i : p > i) v = a[(r0 + i) * rs_a + (r0 + p) * cs_a];
    } else if (i == p) {
      v = T(1);
    }
    L[i][p] = v;
  }
  __syncthreads();
  T x[LEAF];
#pragma unroll
  for (int i = 0; i < LEAF; ++i) x[i] = T(0);
  if (lower) {
#pragma unroll
    for (int i = 0; i < LEAF; ++i) {
      T r = i == j ? T(1) : T(0);
#pragma unroll
      for (int p = 0; p < i; ++p) r = fma(-L[i][p], x[p], r);
      x[i] = r * L[i][i];
    }
  } else {
#pragma unroll
    for (int i = LEAF - 1; i >= 0; --i) {
      T r = i == j ? T(1) : T(0);
#pragma unroll
      for (int p = i + 1; p < LEAF; ++p) r = fma(-L[i][p], x[p], r);
      x[i] = r * L[i][i];
    }
  }
  T *out = inv + (size_t)b * LEAF * LEAF + (size_t)j * LEAF;
#pragma unroll
  for (int i = 0; i < LEAF; ++i) out[i] = x[i];
}

template <typename T>
int launch_inv_diag(int m, const T *a, long rs_a, long cs_a, bool lower, bool unit, T *inv,
                    cudaStream_t s) {
  const int blocks = (int)b200_ceil_div(m, LEAF);
  B200ProfScope prof(sizeof(T) == 4 ? "trsm_inv_s" : "trsm_inv_d", s);
  trsm_inv_diag_kernel<T><<<blocks, LEAF, 0, s>>>(m, a, rs_a, cs_a, lower, unit, inv);
  B200_LAUNCH_CHECK();
  return B200_OK;
}

}  // namespace

namespace {

b200_l3_desc_t plain_gemm_desc(int dtype, int form, int slices) {
  b200_l3_desc_t g;
  memset(&g, 0, sizeof g);
  g.dtype = dtype;
  g.npairs = 1;
  mublis_l3_operand_t gen = {MUBLIS_STRUC_GENERAL, MUBLIS_DENSE, MUBLIS_PACKM_DIAG_NONUNIT};
  g.product.domain.jp = g.product.domain.ji = g.product.domain.pi = MUBLIS_L3_ALL;
  g.product.a = gen;
  g.product.b = gen;
  g.form = form;
  g.slices = slices;
  return g;
}

template <typename T>
int trsm_rec(const b200_trsm_desc_t *d, const T *inv, long r0, long r1) {
  const T *a = (const T *)d->a;
  T *b = (T *)d->b;
  const bool lower = d->uplo == MUBLIS_LOWER;
  long rows = r1 - r0;
  if (rows <= LEAF) {
    // X_b = inv(A_bb) B_b, in place: every CTA of the direct kernel covers
    // all rows of the leaf for its columns (tile height >= LEAF), so it reads
    // its B columns completely before it writes them, and CTAs own disjoint
    // columns.
    b200_l3_desc_t g = plain_gemm_desc(d->dtype, B200_FORM_PLAIN, 0);
    g.m = (int)rows;
    g.n = d->n;
    g.k = (int)rows;
    g.alpha = 1.0;
    g.beta = 0.0;
    g.a[0] = inv + (r0 / LEAF) * LEAF * LEAF;
    g.rs_a[0] = 1;
    g.cs_a[0] = LEAF;
    g.b[0] = b + r0 * d->rs_b;
    g.rs_b[0] = d->rs_b;
    g.cs_b[0] = d->cs_b;
    g.c = b + r0 * d->rs_b;
    g.rs_c = d->rs_b;
    g.cs_c = d->cs_b;
    return b200_gemm_direct_min_rows(&g, LEAF);
  }
  long half = b200_round_up((rows + 1) / 2, LEAF);
  long mid = r0 + half;
  // Rows solved first (src) and rows updated by them (dst).
  long s0 = lower ? r0 : mid, s1 = lower ? mid : r1;
  long t0 = lower ? mid : r0, t1 = lower ? r1 : mid;
  B200_TRY(trsm_rec<T>(d, inv, s0, s1));
  b200_l3_desc_t g = plain_gemm_desc(d->dtype, d->form, d->slices);
  g.m = (int)(t1 - t0);
  g.n = d->n;
  g.k = (int)(s1 - s0);
  g.alpha = -1.0;
  g.beta = 1.0;
  g.a[0] = a + t0 * d->rs_a + s0 * d->cs_a;
  g.rs_a[0] = d->rs_a;
  g.cs_a[0] = d->cs_a;
  g.b[0] = b + s0 * d->rs_b;
  g.rs_b[0] = d->rs_b;
  g.cs_b[0] = d->cs_b;
  g.c = b + t0 * d->rs_b;
  g.rs_c = d->rs_b;
  g.cs_c = d->cs_b;
  // Thin updates (small k) read their operands directly; thick ones go
  // through the packed driver path (and the tensor-core forms).
  B200_TRY(g.k <= 256 ? b200_gemm_direct(&g) : b200_l3_run(&g));
  return trsm_rec<T>(d, inv, t0, t1);
}

template <typename T>
int trsm_solve(const b200_trsm_desc_t *d) {
  cudaStream_t s = b200_cur_stream();
  T *inv = nullptr;
  const long blocks = b200_ceil_div(d->m, LEAF);
  B200_TRY(b200_alloc((void **)&inv, sizeof(T) * blocks * LEAF * LEAF));
  int st = launch_inv_diag<T>(d->m, (const T *)d->a, d->rs_a, d->cs_a, d->uplo == MUBLIS_LOWER,
                              d->unit_diag != 0, inv, s);
  if (st == B200_OK) st = trsm_rec<T>(d, inv, 0, d->m);
  b200_free(inv);
  return st;
}

}  // namespace

extern "C" int b200_trsm_run(const b200_trsm_desc_t *d) {
  if (d->m <= 0 || d->n <= 0) return B200_OK;
  if (d->uplo != MUBLIS_LOWER && d->uplo != MUBLIS_UPPER)
    return b200_set_error(B200_EINVAL, "trsm: uplo must be lower or upper");
  if (d->alpha != 1.0)
    B200_TRY(b200_scale_strided(d->dtype, d->m, d->n, d->alpha, d->b, d->rs_b, d->cs_b,
                                MUBLIS_L3_ALL));
  if (d->dtype == B200_F32) return trsm_solve<float>(d);
  return trsm_solve<double>(d);
}
