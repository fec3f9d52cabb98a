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
#include <cstdlib>
#include <cstring>

#include "kernels.cuh"
#include "tc_common.cuh"
#include "tc_gemm.cuh"

namespace {

// "auto" picks, per call, the fastest form whose error is no worse than the
// plain kernel's: the tensor-core forms pay a split/residue pass and, for
// the integer forms, one int8 product per modulus, so below these sizes
// (crossovers measured on B200) plain wins.  FP32: BF16x6 (3-term split,
// error equal to plain FP32) when min(m, n) and k are >= 512.  FP64: the
// modular Ozaki form with 16 moduli (error ~36x below plain FP64) when
// min(m, n) and k are >= 4096 (at 2048^3 plain is faster, at 4096^3 the
// modular form is 1.8x plain, at 8192^3 2.9x).
int resolve_form(const b200_l3_desc_t *d) {
  int f = d->form == B200_FORM_AUTO ? b200_get_default_form(d->dtype) : d->form;
  if (f == B200_FORM_POLICY) {
    const long m = d->m, n = d->n, k = (long)d->k * d->npairs;
    const long mn = m < n ? m : n;
    if (d->dtype == B200_F32) return mn >= 512 && k >= 512 ? B200_FORM_BF16X6 : B200_FORM_PLAIN;
    return mn >= 4096 && k >= 4096 ? B200_FORM_OZAKI2 : B200_FORM_PLAIN;
  }
  if (d->dtype == B200_F32 && f == B200_FORM_OZAKI) f = B200_FORM_PLAIN;
  if (d->dtype == B200_F64 && (f == B200_FORM_BF16X3 || f == B200_FORM_BF16X6)) f = B200_FORM_PLAIN;
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

int run_dmma(const b200_l3_desc_t *d) {
  cudaStream_t s = b200_cur_stream();
  const long ktot = (long)d->k * d->npairs;
  const long mpad = b200_round_up(d->m, B200_DMMA_TILE);
  const long npad = b200_round_up(d->n, B200_DMMA_TILE);
  const long kpad = b200_round_up(ktot, B200_DMMA_BK);
  void *ap = nullptr, *bp = nullptr;
  B200_TRY(b200_alloc(&ap, sizeof(double) * mpad * kpad));
  int st = b200_alloc(&bp, sizeof(double) * npad * kpad);
  if (st == B200_OK) {
    PackOut oa{ap, kpad, 0, PACK_FRAG64, PACK_COPY, 1, nullptr};
    PackOut ob{bp, kpad, 0, PACK_FRAG64, PACK_COPY, 1, nullptr};
    st = pack_pairs<double>(d, oa, mpad, ob, npad, kpad, s);
  }
  if (st == B200_OK) {
    DmmaGemmArgs g;
    g.ap = (const double *)ap;
    g.bp = (const double *)bp;
    g.kq = kpad / 4;
    g.c = (double *)d->c;
    g.rs_c = d->rs_c;
    g.cs_c = d->cs_c;
    g.m = d->m;
    g.n = d->n;
    g.k = (int)ktot;
    g.tiles_m = (int)(mpad / B200_DMMA_TILE);
    g.tiles_n = (int)(npad / B200_DMMA_TILE);
    g.alpha = d->alpha;
    g.beta = d->beta;
    g.jp = d->product.domain.jp;
    g.ji = d->product.domain.ji;
    g.pi = d->product.domain.pi;
    g.err = b200_device_error_word();
    st = launch_dmma_gemm(g, s);
  }
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
    st = launch_simt_gemm<T>(g, s);
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
  if (form == B200_FORM_BF16X3 || form == B200_FORM_BF16X6) return tc_run_bf16(d, form);
  if (form == B200_FORM_OZAKI || form == B200_FORM_OZAKI2) {
    b200_l3_desc_t e = *d;
    e.form = form;
    if (d->form == B200_FORM_POLICY || (d->form == B200_FORM_AUTO &&
                                        b200_get_default_form(d->dtype) == B200_FORM_POLICY))
      e.slices = form == B200_FORM_OZAKI ? 8 : 0;  // 0: the form's default count
    return tc_run_ozaki(&e);
  }
  if (d->dtype == B200_F32) return run_plain<float>(d);
  return run_plain<double>(d);
}
