// l3.cu -- the device-side generic L3 driver: pack -> contraction ->
// masked epilogue, for every form.  This is what mublis_l3_{s,d}driver (and
// through it GEMM, SYMM, SYRK, SYR2K, TRMM and TRSM's updates) runs.
//
// Reference flow being replaced (frame/l3/l3_driver.c:49-249): a CPU loop
// nest that packs kc x nc panels of B (:133-142) and mc x kc panels of A
// (:152-161), calls the micro-kernel per MR x NR tile and patches edge and
// triangle tiles through a temporary (:192-234).  Here each operand is packed
// once for the whole call (one HBM pass, pack.cu) and the contraction kernel
// tiles the entire output on the device.
#include <cstdint>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "tc_common.cuh"
#include "tc_gemm.cuh"

namespace {

// "auto" picks, per call, the fastest form whose error is no worse than the
// plain kernel's: the tensor-core forms pay a split/residue pass and, for
// the integer forms, one int8 product per modulus, so below these sizes
// (crossovers measured on B200) plain wins.  FP32: BF16x6 (3-term split,
// error equal to plain FP32) when min(m, n) and k are >= 512 (at 256 x 8192
// x 256 plain is faster).  FP64: the modular Ozaki form with 16 moduli (error
// ~36x below plain FP64) when min(m, n) and k are >= 1024 and m n >= 2048^2,
// i.e. at least 64 of its 256 x 256 tiles (measured: 2048^3 0.65 vs 0.71 ms,
// 1024 x 8192 x 1024 0.58 vs 0.76, 2048 x 8192 x 2048 1.28 vs 2.26, 8192^3
// 8.8 vs 32.4; at 1024 x 1024 x 8192 the two tie).
int resolve_form(const b200_l3_desc_t *d) {
  int f = d->form == B200_FORM_AUTO ? b200_get_default_form(d->dtype) : d->form;
  if (f == B200_FORM_POLICY) {
    const long m = d->policy_m > 0 ? d->policy_m : d->m;
    const long n = d->policy_n > 0 ? d->policy_n : d->n;
    const long k = (long)d->k * d->npairs;
    const long mn = m < n ? m : n;
    // FP32: fp16x3 (normwise error ~0.6x plain) where it is at least as fast
    // as bf16x6 (error ~1.0x plain): from 4096 on (at 2048^3 its abs-max
    // pass and slower fp16 MMAs leave it ~10% behind).
    if (d->dtype == B200_F32) {
      if (mn >= 4096 && k >= 2048) return B200_FORM_FP16X3;
      return mn >= 512 && k >= 512 ? B200_FORM_BF16X6 : B200_FORM_PLAIN;
    }
    return mn >= 1024 && k >= 1024 && m * n >= 2048L * 2048 ? B200_FORM_OZAKI2 : B200_FORM_PLAIN;
  }
  if (d->dtype == B200_F32 && f == B200_FORM_OZAKI) f = B200_FORM_PLAIN;
  if (d->dtype == B200_F64 &&
      (f == B200_FORM_BF16X3 || f == B200_FORM_BF16X6 || f == B200_FORM_FP16X3))
    f = B200_FORM_PLAIN;
  return f;
}

// Pack every (A_t, B_t) pair of the descriptor, concatenated along k, into
// the given panel outputs.
template <typename T>
int pack_pairs(const b200_l3_desc_t *d, const PackOut &oa, long mpad, const PackOut &ob,
               long npad, long kpad, cudaStream_t s) {
  const mublis_l3_product_t &pr = d->product;
  for (int t = 0; t < d->npairs; ++t) {
    long kk0 = (long)t * d->k;
    long kk1 = t + 1 == d->npairs ? kpad : kk0 + d->k;
    PackView va{d->a[t], d->rs_a[t], d->cs_a[t], (int)pr.a.struc, (int)pr.a.uplo,
                (int)pr.a.diag, (int)pr.domain.pi};
    PackView vb{d->b[t], d->rs_b[t], d->cs_b[t], (int)pr.b.struc, (int)pr.b.uplo,
                (int)pr.b.diag, (int)pr.domain.jp};
    B200_TRY(launch_pack<T>(va, false, d->m, d->k, mpad, kk0, kk1, oa, s));
    B200_TRY(launch_pack<T>(vb, true, d->n, d->k, npad, kk0, kk1, ob, s));
  }
  return B200_OK;
}

// FP64 GEMM on the tensor pipe (gemm_dmma.cu) unless MUBLIS_B200_DGEMM=simt
// selects the FMA-pipe kernel.
bool use_dmma() {
  static const bool on = [] {
    const char *e = getenv("MUBLIS_B200_DGEMM");
    return !(e && !strcmp(e, "simt"));
  }();
  return on;
}

// A strided FP64 view (rows x cols, element (i, j) at x + i rs + j cs) as a
// TMA source: one stride must be 1 and the other a positive multiple of 2
// elements (16 bytes) at least the unit-stride extent, the base 16-byte
// aligned.  *first_contig: the unit stride runs along the rows index.
bool tma_view_ok(const void *x, long rs, long cs, long rows, long cols, bool *rows_contig) {
  if (((uintptr_t)x & 15) != 0 || rows <= 0 || cols <= 0) return false;
  if (rs == 1 && cs >= rows && cs % 2 == 0) {
    *rows_contig = true;
    return true;
  }
  if (cs == 1 && rs >= cols && rs % 2 == 0) {
    *rows_contig = false;
    return true;
  }
  return false;
}

// Byte interval [lo, hi] spanned by a view with non-negative strides.
void view_span(const void *x, long rs, long cs, long rows, long cols, uintptr_t *lo,
               uintptr_t *hi) {
  *lo = (uintptr_t)x;
  *hi = (uintptr_t)x + sizeof(double) * ((rows - 1) * rs + (cols - 1) * cs + 1) - 1;
}

// The FP64 tensor-pipe kernel can read op(A) and op(B) straight from the
// caller's memory (2-D TMA tiles) instead of packed panels when no element
// needs changing on the way: general operands, no jp / pi mask, every pair
// with the same orientation, a SYR2K's pairs meeting on a k-block boundary,
// and C overlapping no operand (an in-place product must read its operand
// before it is overwritten, which only a copy guarantees).
// MUBLIS_B200_DIRECT=0 keeps the pack pass for every call.
bool dmma_direct(const b200_l3_desc_t *d, DmmaGemmArgs *g) {
  static const bool on = [] {
    const char *e = getenv("MUBLIS_B200_DIRECT");
    return !(e && !strcmp(e, "0"));
  }();
  const mublis_l3_product_t &pr = d->product;
  if (!on || pr.a.struc != MUBLIS_STRUC_GENERAL || pr.b.struc != MUBLIS_STRUC_GENERAL ||
      pr.domain.jp != MUBLIS_L3_ALL || pr.domain.pi != MUBLIS_L3_ALL)
    return false;
  if (d->npairs == 2 && d->k % B200_DMMA_BK != 0) return false;
  if (d->rs_c < 0 || d->cs_c < 0) return false;
  uintptr_t clo, chi;
  view_span(d->c, d->rs_c, d->cs_c, d->m, d->n, &clo, &chi);
  bool a_mc = false, b_kc = false;
  for (int t = 0; t < d->npairs; ++t) {
    bool ac, bc;
    if (!tma_view_ok(d->a[t], d->rs_a[t], d->cs_a[t], d->m, d->k, &ac) ||
        !tma_view_ok(d->b[t], d->rs_b[t], d->cs_b[t], d->k, d->n, &bc))
      return false;
    if (t == 0) {
      a_mc = ac;
      b_kc = bc;
    } else if (ac != a_mc || bc != b_kc) {
      return false;
    }
    uintptr_t lo, hi;
    view_span(d->a[t], d->rs_a[t], d->cs_a[t], d->m, d->k, &lo, &hi);
    if (lo <= chi && clo <= hi) return false;
    view_span(d->b[t], d->rs_b[t], d->cs_b[t], d->k, d->n, &lo, &hi);
    if (lo <= chi && clo <= hi) return false;
  }
  // Tensor maps: op(A) tile 128 (m) x 16 (k), op(B) tile 16 (k) x 128 (n);
  // k innermost tiles are 16 doubles = 128 bytes, 128-byte swizzled.
  memset(g->ta, 0, sizeof g->ta);
  memset(g->tb, 0, sizeof g->tb);
  for (int t = 0; t < d->npairs; ++t) {
    int st = a_mc ? b200_make_tmap_f64(&g->ta[t], d->a[t], d->m, d->k, d->cs_a[t],
                                       B200_DMMA_TILE, B200_DMMA_BK, 0)
                  : b200_make_tmap_f64(&g->ta[t], d->a[t], d->k, d->m, d->rs_a[t],
                                       B200_DMMA_BK, B200_DMMA_TILE, 1);
    if (st == B200_OK)
      st = b_kc ? b200_make_tmap_f64(&g->tb[t], d->b[t], d->k, d->n, d->cs_b[t], B200_DMMA_BK,
                                     B200_DMMA_TILE, 1)
                : b200_make_tmap_f64(&g->tb[t], d->b[t], d->n, d->k, d->rs_b[t],
                                     B200_DMMA_TILE, B200_DMMA_BK, 0);
    if (st != B200_OK) {
      b200_set_error(B200_OK, "");  // not an error: fall back to the pack pass
      return false;
    }
  }
  g->direct = 1;
  g->a_kcontig = !a_mc;
  g->b_kcontig = b_kc;
  g->npairs = d->npairs;
  g->kpair = d->k;
  return true;
}

int run_dmma(const b200_l3_desc_t *d) {
  cudaStream_t s = b200_cur_stream();
  const long ktot = (long)d->k * d->npairs;
  const long mpad = b200_round_up(d->m, B200_DMMA_TILE);
  const long npad = b200_round_up(d->n, B200_DMMA_TILE);
  const long kpad = b200_round_up(ktot, B200_DMMA_BK);
  DmmaGemmArgs g;
  const bool direct = dmma_direct(d, &g);
  void *ap = nullptr, *bp = nullptr;
  int st = B200_OK;
  if (!direct) {
    B200_TRY(b200_alloc(&ap, sizeof(double) * mpad * kpad));
    st = b200_alloc(&bp, sizeof(double) * npad * kpad);
    if (st == B200_OK) {
      PackOut oa{ap, kpad, 0, PACK_FRAG64, PACK_COPY, 1, nullptr};
      PackOut ob{bp, kpad, 0, PACK_FRAG64, PACK_COPY, 1, nullptr};
      st = pack_pairs<double>(d, oa, mpad, ob, npad, kpad, s);
    }
  }
  // Restricted domains: list the tiles that write (ji) with their k-range
  // (jp, pi), heaviest first (the host twin of the kernel's tile_krange).
  const int tiles_m = (int)(mpad / B200_DMMA_TILE), tiles_n = (int)(npad / B200_DMMA_TILE);
  const mublis_l3_domain_t &dom = d->product.domain;
  void *list = nullptr;
  int ntiles = 0;
  if (st == B200_OK &&
      (dom.ji != MUBLIS_L3_ALL || dom.jp != MUBLIS_L3_ALL || dom.pi != MUBLIS_L3_ALL)) {
    std::vector<std::pair<long, int2>> tl;
    const long T = B200_DMMA_TILE, BK = B200_DMMA_BK;
    for (int tm = 0; tm < tiles_m; ++tm)
      for (int tn = 0; tn < tiles_n; ++tn) {
        const long m0 = tm * T, n0 = tn * T;
        if (dom.ji == MUBLIS_L3_LOWER && n0 >= m0 + T) continue;
        if (dom.ji == MUBLIS_L3_UPPER && n0 + T <= m0) continue;
        long kb = 0, ke = ktot;
        if (dom.jp == MUBLIS_L3_LOWER) kb = std::max(kb, n0);
        if (dom.jp == MUBLIS_L3_UPPER) ke = std::min(ke, n0 + T);
        if (dom.pi == MUBLIS_L3_LOWER) ke = std::min(ke, m0 + T);
        if (dom.pi == MUBLIS_L3_UPPER) kb = std::max(kb, m0);
        const long cost = ke > kb ? (ke + BK - 1) / BK - kb / BK : 0;
        tl.push_back({cost, make_int2(tm, tn)});
      }
    std::stable_sort(tl.begin(), tl.end(),
                     [](const std::pair<long, int2> &x, const std::pair<long, int2> &y) {
                       return x.first > y.first;
                     });
    std::vector<int2> flat(tl.size());
    for (size_t i = 0; i < tl.size(); ++i) flat[i] = tl[i].second;
    ntiles = (int)flat.size();
    // The persistent CTAs take tiles round-robin (tile CTA + round * grid);
    // with the list heaviest first, reversing every other round ("snake")
    // evens out each CTA's total instead of giving CTA 0 the heaviest tile
    // of every round.
    const size_t grid = (size_t)std::min(ntiles, b200_sm_count());
    for (size_t r0 = grid; grid > 0 && r0 < flat.size(); r0 += 2 * grid)
      std::reverse(flat.begin() + r0, flat.begin() + std::min(flat.size(), r0 + grid));
    st = b200_alloc(&list, sizeof(int2) * (ntiles > 0 ? ntiles : 1));
    if (st == B200_OK && ntiles > 0 &&
        cudaMemcpyAsync(list, flat.data(), sizeof(int2) * ntiles, cudaMemcpyHostToDevice, s) !=
            cudaSuccess)
      st = b200_set_error(B200_ECUDA, "dgemm: tile list upload failed");
  }
  // Split-K from the whole call's shape (column panels carry the call's m
  // and n), so panels split their tiles' k ranges as the whole call does.
  const int S = b200_split_for(d->policy_m > 0 ? d->policy_m : d->m,
                               d->policy_n > 0 ? d->policy_n : d->n, ktot, B200_DMMA_TILE,
                               B200_DMMA_TILE, B200_DMMA_BK, {dom.jp, dom.ji, dom.pi},
                               b200_sm_count(), 8.0);  // 128 KB of partials per split unit
  const long sched_tiles = list ? ntiles : (long)tiles_m * tiles_n;
  void *split_ws = nullptr;
  if (st == B200_OK && S > 1) {
    const size_t ints = b200_round_up(sizeof(int) * sched_tiles * 8, 256);
    st = b200_alloc(&split_ws, ints + sizeof(double) * (size_t)sched_tiles * S * 64 * 256);
    if (st == B200_OK && cudaMemsetAsync(split_ws, 0, ints, s) != cudaSuccess)
      st = b200_set_error(B200_ECUDA, "dgemm: split-K counters");
  }
  if (st == B200_OK && (list == nullptr || ntiles > 0)) {
    g.ap = (const double *)ap;
    g.bp = (const double *)bp;
    g.kq = kpad / 4;
    g.c = (double *)d->c;
    g.rs_c = d->rs_c;
    g.cs_c = d->cs_c;
    g.m = d->m;
    g.n = d->n;
    g.k = (int)ktot;
    g.tiles_m = tiles_m;
    g.tiles_n = tiles_n;
    g.tile_list = (const int2 *)list;
    g.ntiles = ntiles;
    g.alpha = d->alpha;
    g.beta = d->beta;
    g.jp = d->product.domain.jp;
    g.ji = d->product.domain.ji;
    g.pi = d->product.domain.pi;
    g.err = b200_device_error_word();
    g.wait_ns = B200_WAIT_NS;
    g.stall = 0;
    if (const unsigned long long limit = b200_take_test_stall()) {
      g.wait_ns = limit;
      g.stall = 1;
    }
    g.splits = S;
    if (S > 1) {
      g.arrivals = (int *)split_ws;
      g.partials = (double *)((char *)split_ws +
                              b200_round_up(sizeof(int) * sched_tiles * 8, 256));
    }
    st = launch_dmma_gemm(g, s);
  }
  b200_free(split_ws);
  b200_free(list);
  b200_free(ap);
  b200_free(bp);
  return st;
}

template <typename T>
int run_plain(const b200_l3_desc_t *d) {
  if (sizeof(T) == 8 && use_dmma()) return run_dmma(d);
  using C = SimtConfig<T>;
  cudaStream_t s = b200_cur_stream();
  const long ktot = (long)d->k * d->npairs;
  const long mpad = b200_round_up(d->m, C::BM), npad = b200_round_up(d->n, C::BN);
  const long kpad = b200_round_up(ktot, C::BK);
  void *ap = nullptr, *bp = nullptr;
  B200_TRY(b200_alloc(&ap, sizeof(T) * mpad * kpad));
  int st = b200_alloc(&bp, sizeof(T) * npad * kpad);
  if (st == B200_OK) {
    PackOut oa{ap, mpad, 0, PACK_MN_MAJOR, PACK_COPY, 1, nullptr};
    PackOut ob{bp, npad, 0, PACK_MN_MAJOR, PACK_COPY, 1, nullptr};
    st = pack_pairs<T>(d, oa, mpad, ob, npad, kpad, s);
  }
  if (st == B200_OK) {
    SimtGemmArgs<T> g;
    g.ap = (const T *)ap;
    g.bp = (const T *)bp;
    g.lda = mpad;
    g.ldb = npad;
    g.c = (T *)d->c;
    g.rs_c = d->rs_c;
    g.cs_c = d->cs_c;
    g.m = d->m;
    g.n = d->n;
    g.k = (int)ktot;
    g.alpha = (T)d->alpha;
    g.beta = (T)d->beta;
    g.jp = d->product.domain.jp;
    g.ji = d->product.domain.ji;
    g.pi = d->product.domain.pi;
    const SimtPolicy pol = {d->policy_m > 0 ? d->policy_m : d->m,
                            d->policy_n > 0 ? d->policy_n : d->n};
    st = launch_simt_gemm<T>(g, s, &pol);
  }
  b200_free(ap);
  b200_free(bp);
  return st;
}

}  // namespace

extern "C" int b200_scale_strided(int dtype, int m, int n, double beta, void *c, long rs, long cs,
                                  mublis_l3_relation_t ji) {
  cudaStream_t s = b200_cur_stream();
  if (dtype == B200_F32) return launch_scale<float>(m, n, (float)beta, (float *)c, rs, cs, ji, s);
  return launch_scale<double>(m, n, beta, (double *)c, rs, cs, ji, s);
}

extern "C" int b200_l3_run(const b200_l3_desc_t *d) {
  if (d->m <= 0 || d->n <= 0) return B200_OK;
  if (d->npairs < 1 || d->npairs > 2) return b200_set_error(B200_EINVAL, "l3: npairs");
  // alpha == 0 (or no k): beta-scale the written part only, never touching
  // A or B (l3_driver.c:104,123).
  if (d->alpha == 0.0 || d->k <= 0)
    return b200_scale_strided(d->dtype, d->m, d->n, d->beta, d->c, d->rs_c, d->cs_c,
                              d->product.domain.ji);
  const int form = resolve_form(d);
  if (form == B200_FORM_BF16X3 || form == B200_FORM_BF16X6 || form == B200_FORM_FP16X3)
    return tc_run_bf16(d, form);
  if (form == B200_FORM_OZAKI || form == B200_FORM_OZAKI2) {
    b200_l3_desc_t e = *d;
    e.form = form;
    if (d->form == B200_FORM_POLICY || (d->form == B200_FORM_AUTO &&
                                        b200_get_default_form(d->dtype) == B200_FORM_POLICY))
      e.slices = form == B200_FORM_OZAKI ? 8 : 0;  // 0: the form's default count
    // "ozaki2@<target>": the modulus count measured for the target error
    // (cached per precision, k bucket and target).
    const double target = b200_get_default_target(d->dtype);
    if (form == B200_FORM_OZAKI2 && d->form == B200_FORM_AUTO && target > 0 && d->slices == 0 &&
        b200_get_default_form(d->dtype) == B200_FORM_OZAKI2 &&
        b200_get_default_slices(d->dtype) == 0)
      B200_TRY(b200_ozaki2_choice(&e, target, &e.slices, nullptr, 0));
    return tc_run_ozaki(&e);
  }
  if (d->dtype == B200_F32) return run_plain<float>(d);
  return run_plain<double>(d);
}
