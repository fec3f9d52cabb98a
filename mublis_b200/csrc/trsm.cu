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
//   * FP64 leaves (512 rows) are solved by the fused GEMMTRSM kernel
//     (trsm_leaf.cu): diagonal 16 x 16 blocks in shared memory, the updates
//     between them on the FP64 tensor pipe, every right-hand side of the
//     chain in one launch;
//   * FP32 leaves are the 512 x 512 (1024 x 1024 for large solves) diagonal
//     blocks, inverted up front: one launch inverts every 64 x 64 diagonal
//     block by substitution against the reciprocal diagonal (computed once
//     and multiplied -- never divided -- as the reference does), then
//     doubling steps of two batched (grouped) GEMM launches each build the
//     128-, 256-, 512- (and 1024-) blocks,
//     inv([A11 0; A21 A22]) = [inv11 0; -inv22 A21 inv11  inv22];
//   * each leaf solve is then X_b = inv(A_bb) B_b, one triangular product
//     over all right-hand sides (plain FP64/FP32: the diagonal blocks never
//     use an emulated form), and every update is a GEMM of k >= 512 on the
//     packed path (and the caller's form).  512-row leaves give those GEMMs
//     at least 128 output tiles of 128 x 128 for 148 SMs (256-row leaves
//     gave 64);
//   * the unit diagonal and the unstored triangle are never read.
// alpha is applied once up front (the reference's alpha_eff on the first
// block, trsm.c:96-97).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "kernels.cuh"

namespace {

constexpr int LEAF = 64;  // diagonal blocks inverted by substitution

// Order of the inverted diagonal blocks the solve uses (its leaves): 512, or
// 1024 for large solves.  A leaf product inv(A_bb) B_b over n right-hand
// sides is a triangular GEMM of 512 (1024) rows: 1024-row leaves give it
// 256 output tiles of 128 x 128 instead of 128 (148 SMs) and remove the
// level of 512-row updates below them, for one more doubling step (about
// m * 512^2 extra flops).  With few right-hand sides that doubling step
// would cost more than it saves, so 1024 is used only from m >= 4096 and
// n >= 2048.
int leaf_order(long m, long n) {
  // MUBLIS_B200_TRSM_LEAF=<256|512|1024> fixes it (tuning).
  static const int forced = [] {
    const char *e = getenv("MUBLIS_B200_TRSM_LEAF");
    const int v = e ? atoi(e) : 0;
    return v == 256 || v == 512 || v == 1024 ? v : 0;
  }();
  if (forced) return forced;
  return m >= 4096 && n >= 2048 ? 1024 : 512;
}

// Leaves: FP64 solves use the fused leaf kernel (trsm_leaf.cu), FP32 solves
// the inverted diagonal blocks applied as products; MUBLIS_B200_TRSM=fused /
// inverse selects one for both.  Measured at n = 4096 (device operands):
// DTRSM 22.4 TF/s fused vs 20.3 inverse (the leaf's updates run on the FP64
// tensor pipe, and it executes the triangle's flops only, not the 1.25 to 2x
// of a product with the inverse); STRSM 31.0 fused vs 33.3 inverse (FP32 has
// no tensor-pipe form, and the inverse products run at the SIMT GEMM's rate).
bool fused_leaves(int dtype) {
  static const int forced = [] {
    const char *e = getenv("MUBLIS_B200_TRSM");
    if (e && !strcmp(e, "inverse")) return 0;
    if (e && !strcmp(e, "fused")) return 1;
    return -1;
  }();
  return forced >= 0 ? forced == 1 : dtype == B200_F64;
}

// One CTA per LEAF block: thread j computes column j of the inverse of the
// block's (lower or upper) triangle by substitution, L x = e_j.  Rows past
// the matrix order are padded with the identity.  Output: big block
// b / per_big (per_big = big / LEAF) is a big x big column-major matrix at
// inv + (b / per_big) * big * big (zeroed beforehand); LEAF block b lands on
// its diagonal at offset (b % per_big) * LEAF.
template <typename T>
__global__ void __launch_bounds__(LEAF) trsm_inv_diag_kernel(int m, const T *a, long rs_a,
                                                              long cs_a, bool lower, bool unit,
                                                              T *inv, int big) {
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
  const int per_big = big / LEAF;
  const size_t off = (size_t)(b % per_big) * LEAF;
  T *out = inv + (size_t)(b / per_big) * big * big + off * (big + 1) + (size_t)j * big;
#pragma unroll
  for (int i = 0; i < LEAF; ++i) out[i] = x[i];
}

template <typename T>
int launch_inv_diag(int m, const T *a, long rs_a, long cs_a, bool lower, bool unit, T *inv,
                    int big, cudaStream_t s) {
  const int blocks = (int)b200_ceil_div(m, LEAF);
  B200ProfScope prof(sizeof(T) == 4 ? "trsm_inv_s" : "trsm_inv_d", s);
  trsm_inv_diag_kernel<T><<<blocks, LEAF, 0, s>>>(m, a, rs_a, cs_a, lower, unit, inv, big);
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

// Doubling: with the inverses of the h-blocks on the diagonal of every big
// block, fill in the off-diagonal h x h block of every 2h-block:
//   lower  X21 = -inv22 (A21 inv11),   upper  X12 = -inv11 (A12 inv22),
// as two grouped launches (the products into `tmp`, then into `inv`).  A
// pair whose second half is cut by the matrix order uses only its valid
// m2 rows/columns; the identity padding makes the rest already correct.
template <typename T>
int grow_inverse(const b200_trsm_desc_t *d, T *inv, T *tmp, const long big, cudaStream_t s) {
  const T *a = (const T *)d->a;
  const bool lower = d->uplo == MUBLIS_LOWER;
  const long m = d->m;
  for (long h = LEAF; h < big; h *= 2) {
    std::vector<b200_l3_desc_t> g1, g2;
    for (long r0 = 0; r0 + h < m; r0 += 2 * h) {
      const int m2 = (int)std::min(h, m - r0 - h);
      T *blk = inv + (r0 / big) * big * big;
      const long o1 = r0 % big, o2 = o1 + h;
      const T *inv11 = blk + o1 * (big + 1), *inv22 = blk + o2 * (big + 1);
      T *t = tmp + (r0 / (2 * h)) * h * h;
      b200_l3_desc_t p = plain_gemm_desc(d->dtype, B200_FORM_PLAIN, 0);
      b200_l3_desc_t q = p;
      p.alpha = 1.0;
      q.alpha = -1.0;
      p.beta = q.beta = 0.0;
      if (lower) {  // T (m2 x h) = A21 inv11;  X21 = -inv22[m2 x m2] T
        p.m = m2, p.n = (int)h, p.k = (int)h;
        p.a[0] = a + (r0 + h) * d->rs_a + r0 * d->cs_a, p.rs_a[0] = d->rs_a, p.cs_a[0] = d->cs_a;
        p.b[0] = inv11, p.rs_b[0] = 1, p.cs_b[0] = big;
        q.m = m2, q.n = (int)h, q.k = m2;
        q.a[0] = inv22, q.rs_a[0] = 1, q.cs_a[0] = big;
        q.c = blk + o2 + o1 * big;
      } else {  // T (h x m2) = A12 inv22[m2 x m2];  X12 = -inv11 T
        p.m = (int)h, p.n = m2, p.k = m2;
        p.a[0] = a + r0 * d->rs_a + (r0 + h) * d->cs_a, p.rs_a[0] = d->rs_a, p.cs_a[0] = d->cs_a;
        p.b[0] = inv22, p.rs_b[0] = 1, p.cs_b[0] = big;
        q.m = (int)h, q.n = m2, q.k = (int)h;
        q.a[0] = inv11, q.rs_a[0] = 1, q.cs_a[0] = big;
        q.c = blk + o1 + o2 * big;
      }
      p.c = t, p.rs_c = 1, p.cs_c = h;
      q.b[0] = t, q.rs_b[0] = 1, q.cs_b[0] = h;
      q.rs_c = 1, q.cs_c = big;
      g1.push_back(p);
      g2.push_back(q);
    }
    if (g1.empty()) break;
    std::vector<const b200_l3_desc_t *> p1, p2;
    for (size_t i = 0; i < g1.size(); ++i) {
      p1.push_back(&g1[i]);
      p2.push_back(&g2[i]);
    }
    B200_TRY(b200_grouped_gemm_async(d->dtype, p1.data(), (int)p1.size(), s));
    B200_TRY(b200_grouped_gemm_async(d->dtype, p2.data(), (int)p2.size(), s));
  }
  return B200_OK;
}

// One L3 product per column chain: chain c runs on streams[c] (the
// thread's stream is overridden for it), so chains are enqueued in lockstep.
struct Chains {
  const b200_trsm_desc_t *d[2];
  cudaStream_t streams[2];
  int count;
};

template <typename Build>
int for_each_chain(const Chains &ch, Build build) {
  for (int c = 0; c < ch.count; ++c) {
    b200_l3_desc_t g = build(*ch.d[c]);
    void *prev = b200_override_stream((void *)ch.streams[c]);
    const int st = b200_l3_run(&g);
    b200_override_stream(prev);
    B200_TRY(st);
  }
  return B200_OK;
}

// Inverted diagonal blocks of one triangle (FP32: the leaves of the solve,
// applied as products), or (FP64) the packed leaves of the fused
// GEMMTRSM kernel (trsm_leaf.cu).
struct TrsmPrep {
  void *inv;
  long big;
  void *leaf;
};

template <typename T>
int trsm_rec(const Chains &ch, const TrsmPrep *prep, long r0, long r1) {
  const b200_trsm_desc_t &d0 = *ch.d[0];
  const bool lower = d0.uplo == MUBLIS_LOWER;
  const T *inv = (const T *)prep->inv;
  const long big = prep->big;
  long rows = r1 - r0;
  if (rows <= big && prep->leaf) {
    // Fused leaf: the diagonal blocks solved in shared memory, the updates
    // between them on the tensor pipe, every right-hand side of the chain.
    for (int c = 0; c < ch.count; ++c) {
      const b200_trsm_desc_t &d = *ch.d[c];
      T *b = (T *)d.b;
      const T *pack = (const T *)prep->leaf + (r0 / big) * b200_trsm_leaf_stride();
      static_assert(sizeof(T) == 4 || sizeof(T) == 8, "FP32 / FP64");
      T *first = lower ? b + r0 * d.rs_b : b + (r1 - 1) * d.rs_b;
      void *prev = b200_override_stream((void *)ch.streams[c]);
      const int st = b200_trsm_leaf_solve(d.dtype, pack, (int)rows, first,
                                          lower ? d.rs_b : -d.rs_b, d.cs_b, d.n);
      b200_override_stream(prev);
      B200_TRY(st);
    }
    return B200_OK;
  }
  if (rows <= big) {
    // X_b = inv(A_bb) B_b in place: the packed path packs B_b before the
    // product writes it.  Plain precision: the diagonal-block solve is FP64
    // (FP32) whatever form the updates use.  inv(A_bb) is triangular like
    // A_bb, so it goes in as a triangular operand with the matching k range
    // per row tile (pi LOWER / UPPER): the zero tiles are not multiplied.
    return for_each_chain(ch, [&](const b200_trsm_desc_t &d) {
      T *b = (T *)d.b;
      b200_l3_desc_t g = plain_gemm_desc(d.dtype, B200_FORM_PLAIN, 0);
      // The whole call's n: a column panel (or chain) of a larger solve then
      // schedules (splits) the product as the whole call would, so every
      // column gets the same bits either way.
      g.policy_n = d.policy_n;
      g.product.domain.pi = lower ? MUBLIS_L3_LOWER : MUBLIS_L3_UPPER;
      g.product.a.struc = MUBLIS_STRUC_TRIANGULAR;
      g.product.a.uplo = d.uplo;
      g.m = (int)rows;
      g.n = d.n;
      g.k = (int)rows;
      g.alpha = 1.0;
      g.beta = 0.0;
      g.a[0] = inv + (r0 / big) * big * big;
      g.rs_a[0] = 1;
      g.cs_a[0] = big;
      g.b[0] = b + r0 * d.rs_b;
      g.rs_b[0] = d.rs_b;
      g.cs_b[0] = d.cs_b;
      g.c = b + r0 * d.rs_b;
      g.rs_c = d.rs_b;
      g.cs_c = d.cs_b;
      return g;
    });
  }
  long half = b200_round_up((rows + 1) / 2, big);
  long mid = r0 + half;
  // Rows solved first (src) and rows updated by them (dst).
  long s0 = lower ? r0 : mid, s1 = lower ? mid : r1;
  long t0 = lower ? mid : r0, t1 = lower ? r1 : mid;
  B200_TRY(trsm_rec<T>(ch, prep, s0, s1));
  B200_TRY(for_each_chain(ch, [&](const b200_trsm_desc_t &d) {
    const T *a = (const T *)d.a;
    T *b = (T *)d.b;
    b200_l3_desc_t g = plain_gemm_desc(d.dtype, d.form, d.slices);
    g.policy_n = d.policy_n;
    g.m = (int)(t1 - t0);
    g.n = d.n;
    g.k = (int)(s1 - s0);
    g.alpha = -1.0;
    g.beta = 1.0;
    g.a[0] = a + t0 * d.rs_a + s0 * d.cs_a;
    g.rs_a[0] = d.rs_a;
    g.cs_a[0] = d.cs_a;
    g.b[0] = b + s0 * d.rs_b;
    g.rs_b[0] = d.rs_b;
    g.cs_b[0] = d.cs_b;
    g.c = b + t0 * d.rs_b;
    g.rs_c = d.rs_b;
    g.cs_c = d.cs_b;
    return g;
  }));
  return trsm_rec<T>(ch, prep, t0, t1);
}

// Pack every leaf of op(A) for the fused kernel (reciprocal diagonal; FP64
// panel blocks in MMA fragment order, FP32 column-major).
int build_leaves(const b200_trsm_desc_t *d, TrsmPrep *p) {
  const long leaves = b200_ceil_div(d->m, b200_trsm_leaf_rows());
  const size_t elt = d->dtype == B200_F32 ? sizeof(float) : sizeof(double);
  void *pack = nullptr;
  B200_TRY(b200_alloc(&pack, elt * leaves * b200_trsm_leaf_stride()));
  const int st = b200_trsm_leaf_pack(d->dtype, d->a, d->rs_a, d->cs_a, d->m,
                                     d->uplo == MUBLIS_LOWER, d->unit_diag != 0, pack);
  if (st != B200_OK) {
    b200_free(pack);
    return st;
  }
  p->inv = nullptr;
  p->big = b200_trsm_leaf_rows();
  p->leaf = pack;
  return B200_OK;
}

template <typename T>
int build_inverse(const b200_trsm_desc_t *d, TrsmPrep *p) {
  if (fused_leaves(d->dtype)) return build_leaves(d, p);
  cudaStream_t s = b200_cur_stream();
  T *inv = nullptr, *tmp = nullptr;
  const long big = leaf_order(d->m, d->policy_n > 0 ? d->policy_n : d->n);
  const long bigs = b200_ceil_div(d->m, big);
  B200_TRY(b200_alloc((void **)&inv, sizeof(T) * bigs * big * big));
  int st = b200_alloc((void **)&tmp, sizeof(T) * bigs * big * big / 2);
  if (st == B200_OK && cudaMemsetAsync(inv, 0, sizeof(T) * bigs * big * big, s) != cudaSuccess)
    st = b200_set_error(B200_ECUDA, "trsm: memset failed");
  if (st == B200_OK)
    st = launch_inv_diag<T>(d->m, (const T *)d->a, d->rs_a, d->cs_a, d->uplo == MUBLIS_LOWER,
                            d->unit_diag != 0, inv, (int)big, s);
  if (st == B200_OK) st = grow_inverse<T>(d, inv, tmp, big, s);
  b200_free(tmp);
  if (st != B200_OK) {
    b200_free(inv);
    return st;
  }
  p->inv = inv;
  p->big = big;
  p->leaf = nullptr;
  return B200_OK;
}

template <typename T>
int trsm_solve(const b200_trsm_desc_t *d) {
  cudaStream_t s = b200_cur_stream();
  TrsmPrep own = {nullptr, 0, nullptr};
  const TrsmPrep *prep = (const TrsmPrep *)d->prep;
  if (!prep) {
    B200_TRY(build_inverse<T>(d, &own));
    prep = &own;
  }
  int st = B200_OK;
  if (st == B200_OK) {
    // The right-hand sides are independent: a large solve runs its two
    // column halves as two chains of the same launches on two streams, so
    // one half's kernels fill the wave tails of the other's (every column
    // is computed exactly as in one chain).
    cudaStream_t s2 = d->n >= 2048 && d->m >= 2048 ? (cudaStream_t)b200_aux_stream() : nullptr;
    if (s2) {
      b200_trsm_desc_t h0 = *d, h1 = *d;
      const long half = b200_round_up((d->n + 1) / 2, 128);
      h0.policy_n = h1.policy_n = d->policy_n > 0 ? d->policy_n : d->n;
      h0.n = (int)half;
      h1.n = (int)(d->n - half);
      h1.b = (T *)d->b + half * d->cs_b;
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      if (cudaEventCreateWithFlags(&e0, cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&e1, cudaEventDisableTiming) != cudaSuccess ||
          cudaEventRecord(e0, s) != cudaSuccess || cudaStreamWaitEvent(s2, e0, 0) != cudaSuccess)
        st = b200_set_error(B200_ECUDA, "trsm: stream fork failed");
      if (st == B200_OK) {
        const Chains ch = {{&h0, &h1}, {s, s2}, 2};
        st = trsm_rec<T>(ch, prep, 0, d->m);
      }
      // Join even after a failure, so nothing of the second chain is left
      // running on the scratch freed below.
      if (e1 && (cudaEventRecord(e1, s2) != cudaSuccess ||
                 cudaStreamWaitEvent(s, e1, 0) != cudaSuccess) && st == B200_OK)
        st = b200_set_error(B200_ECUDA, "trsm: stream join failed");
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
    } else {
      const Chains ch = {{d, nullptr}, {s, nullptr}, 1};
      st = trsm_rec<T>(ch, prep, 0, d->m);
    }
  }
  b200_free(own.inv);
  b200_free(own.leaf);
  return st;
}

}  // namespace

extern "C" int b200_trsm_prepare(const b200_trsm_desc_t *d, void **prep) {
  *prep = nullptr;
  if (d->m <= 0) return B200_OK;
  if (d->uplo != MUBLIS_LOWER && d->uplo != MUBLIS_UPPER)
    return b200_set_error(B200_EINVAL, "trsm: uplo must be lower or upper");
  TrsmPrep *p = new TrsmPrep{nullptr, 0, nullptr};
  const int st = d->dtype == B200_F32 ? build_inverse<float>(d, p) : build_inverse<double>(d, p);
  if (st != B200_OK) {
    delete p;
    return st;
  }
  *prep = p;
  return B200_OK;
}

extern "C" void b200_trsm_release(void *prep) {
  TrsmPrep *p = (TrsmPrep *)prep;
  if (!p) return;
  b200_free(p->inv);  // stream-ordered after the panels on this stream
  b200_free(p->leaf);
  delete p;
}

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
