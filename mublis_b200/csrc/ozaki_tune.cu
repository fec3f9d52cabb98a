// ozaki_tune.cu -- the modulus count of the modular Ozaki form, chosen by
// measurement for a stated target error.
//
// The modular form (tc_gemm.cu) keeps pa + pb bits of each scaled input,
// where k 2^(pa+pb) must fit under half the product M of its N moduli: each
// modulus adds about 8 bits and one int8 product per k-block, so the
// fastest form that meets an error target is the one with the fewest moduli
// that meets it.  How many that is depends on k and on the data (a row
// whose elements span many binades loses the small ones' low bits to the
// row's scaling), so it is measured rather than assumed:
//   * a calibration block of the call itself -- the leading 256 x 256 of C
//     (fewer if C is smaller), i.e. the first 256 rows of op(A) and columns
//     of op(B) over the whole k, with the call's operand structures and
//     domain -- is computed by a compensated dot product on the device
//     (Ogita, Rump and Oishi's Dot2: TwoProduct by FMA and TwoSum, about
//     twice working precision) as the reference;
//   * the form runs on the same block with N = 6 .. 16 moduli (FP32:
//     6 .. 8) from the fewest up, and the first N whose normwise error
//     ||C_N - C_ref||_F / (||A_blk||_F ||B_blk||_F) is within the target is
//     kept (16 if none is);
//   * the choice is cached per (precision, power-of-two bucket of k,
//     target) and saved with the tuned-tile table.
// The form "ozaki2@<target>" makes every call of that precision use the
// cached choice, calibrating on the first call of a new key.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "kernels.cuh"
#include "tc_gemm.cuh"

namespace {

constexpr int CAL = 256;  // calibration block edge

// Dot2 (Ogita, Rump and Oishi 2005) of row i of op(A) and column j of op(B)
// over every pair of the descriptor (concatenated along k); thread (i, 0) and
// (0, j) also return the row's / column's sum of squares.
template <typename T>
__global__ void dot2_block_kernel(PackView va0, PackView va1, PackView vb0, PackView vb1, int npairs,
                                  int m, int n, long k, double *hi, double *lo, double *rsq,
                                  double *csq) {
  const int i = blockIdx.y * blockDim.y + threadIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m || j >= n) return;
  double s = 0.0, c = 0.0, ra = 0.0, cb = 0.0;
  for (int t = 0; t < npairs; ++t) {
    const PackView &va = t ? va1 : va0;
    const PackView &vb = t ? vb1 : vb0;
    for (long p = 0; p < k; ++p) {
      const double a = (double)load_logical<T>(va, i, p);
      const double b = (double)load_logical<T>(vb, p, j);
      const double prod = a * b;
      const double perr = fma(a, b, -prod);  // TwoProduct
      const double s2 = s + prod;            // TwoSum
      const double z = s2 - s;
      const double serr = (s - (s2 - z)) + (prod - z);
      s = s2;
      c += perr + serr;
      if (j == 0) ra = fma(a, a, ra);
      if (i == 0) cb = fma(b, b, cb);
    }
  }
  const double h = s + c;
  hi[(long)i * n + j] = h;
  lo[(long)i * n + j] = c - (h - s);
  if (j == 0) rsq[i] = ra;
  if (i == 0) csq[j] = cb;
}

std::mutex g_mu;
// (fp64, k bucket, target bits) -> (moduli, measured error)
std::map<std::tuple<int, int, unsigned long long>, std::pair<int, double>> g_choice;

int k_bucket(long k) {
  int b = 0;
  while ((1L << b) < k) ++b;
  return b;
}

unsigned long long bits_of(double x) {
  unsigned long long u;
  memcpy(&u, &x, sizeof u);
  return u;
}

template <typename T>
int calibrate(const b200_l3_desc_t *d, double target, int *moduli, double *measured) {
  cudaStream_t s = b200_cur_stream();
  const int cm = d->m < CAL ? d->m : CAL, cn = d->n < CAL ? d->n : CAL;
  const long k = d->k;
  const mublis_l3_product_t &pr = d->product;
  PackView va[2], vb[2];
  for (int t = 0; t < 2; ++t) {
    const int u = t < d->npairs ? t : 0;
    va[t] = PackView{d->a[u], d->rs_a[u], d->cs_a[u], (int)pr.a.struc, (int)pr.a.uplo,
                     (int)pr.a.diag, (int)pr.domain.pi};
    vb[t] = PackView{d->b[u], d->rs_b[u], d->cs_b[u], (int)pr.b.struc, (int)pr.b.uplo,
                     (int)pr.b.diag, (int)pr.domain.jp};
  }
  const size_t cells = (size_t)cm * cn;
  void *ws = nullptr;
  B200_TRY(b200_alloc(&ws, sizeof(double) * (3 * cells + cm + cn)));
  double *hi = (double *)ws, *lo = hi + cells, *cal = lo + cells, *rsq = cal + cells,
         *csq = rsq + cm;
  int st = B200_OK;
  {
    dim3 blk(32, 8), grid((unsigned)b200_ceil_div(cn, 32), (unsigned)b200_ceil_div(cm, 8));
    B200ProfScope prof("ozaki2_tune_dot2", s);
    dot2_block_kernel<T><<<grid, blk, 0, s>>>(va[0], va[1], vb[0], vb[1], d->npairs, cm, cn, k,
                                              hi, lo, rsq, csq);
    if (cudaGetLastError() != cudaSuccess) st = b200_set_error(B200_ECUDA, "ozaki2 tune: launch");
  }
  std::vector<double> h_hi(cells), h_lo(cells), h_c(cells), h_r(cm), h_cq(cn);
  if (st == B200_OK &&
      (cudaMemcpyAsync(h_hi.data(), hi, sizeof(double) * cells, cudaMemcpyDeviceToHost, s) !=
           cudaSuccess ||
       cudaMemcpyAsync(h_lo.data(), lo, sizeof(double) * cells, cudaMemcpyDeviceToHost, s) !=
           cudaSuccess ||
       cudaMemcpyAsync(h_r.data(), rsq, sizeof(double) * cm, cudaMemcpyDeviceToHost, s) !=
           cudaSuccess ||
       cudaMemcpyAsync(h_cq.data(), csq, sizeof(double) * cn, cudaMemcpyDeviceToHost, s) !=
           cudaSuccess ||
       cudaStreamSynchronize(s) != cudaSuccess))
    st = b200_set_error(B200_ECUDA, "ozaki2 tune: reference copy");
  long double na = 0, nb = 0;
  for (int i = 0; i < cm; ++i) na += h_r[i];
  for (int j = 0; j < cn; ++j) nb += h_cq[j];
  const long double den = sqrtl(na) * sqrtl(nb);
  const bool F64 = sizeof(T) == 8;
  const int lo_n = 6, hi_n = F64 ? B200_MAX_MODULI : 8;
  int chosen = hi_n;
  double chosen_err = -1.0;
  for (int N = lo_n; N <= hi_n && st == B200_OK; ++N) {
    b200_l3_desc_t e = *d;
    e.m = cm;
    e.n = cn;
    e.alpha = 1.0;
    e.beta = 0.0;
    e.c = cal;  // row-major: element (i, j) at i * cn + j, as the reference
    e.rs_c = cn;
    e.cs_c = 1;
    e.form = B200_FORM_OZAKI2;
    e.slices = N;
    std::vector<float> h_cf;  // FP32 calls write FP32 results (into the same buffer)
    const int rs = tc_run_ozaki(&e);
    if (rs == B200_EINVAL) continue;  // too few moduli for this k
    if (rs != B200_OK) {
      st = rs;
      break;
    }
    long double num = 0;
    if (F64) {
      if (cudaMemcpyAsync(h_c.data(), cal, sizeof(double) * cells, cudaMemcpyDeviceToHost, s) !=
              cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        st = b200_set_error(B200_ECUDA, "ozaki2 tune: result copy");
        break;
      }
      for (size_t q = 0; q < cells; ++q) {
        const long double dlt = ((long double)h_c[q] - h_hi[q]) - h_lo[q];
        num += dlt * dlt;
      }
    } else {
      h_cf.resize(cells);
      if (cudaMemcpyAsync(h_cf.data(), cal, sizeof(float) * cells, cudaMemcpyDeviceToHost, s) !=
              cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess) {
        st = b200_set_error(B200_ECUDA, "ozaki2 tune: result copy");
        break;
      }
      for (size_t q = 0; q < cells; ++q) {
        const long double dlt = ((long double)h_cf[q] - h_hi[q]) - h_lo[q];
        num += dlt * dlt;
      }
    }
    const double err = den > 0 ? (double)(sqrtl(num) / den) : 0.0;
    chosen = N;
    chosen_err = err;
    if (err <= target) break;
  }
  b200_free(ws);
  if (st != B200_OK) return st;
  *moduli = chosen;
  *measured = chosen_err;
  return B200_OK;
}

}  // namespace

int b200_ozaki2_choice(const b200_l3_desc_t *d, double target, int *moduli, double *measured,
                       int force) {
  if (!(target > 0)) return b200_set_error(B200_EINVAL, "ozaki2 tune: target must be > 0");
  const auto key = std::make_tuple(d->dtype == B200_F64 ? 1 : 0,
                                   k_bucket((long)d->k * d->npairs), bits_of(target));
  if (!force) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_choice.find(key);
    if (it != g_choice.end()) {
      *moduli = it->second.first;
      if (measured) *measured = it->second.second;
      return B200_OK;
    }
  }
  double err = 0;
  const int st = d->dtype == B200_F64 ? calibrate<double>(d, target, moduli, &err)
                                      : calibrate<float>(d, target, moduli, &err);
  if (st != B200_OK) return st;
  if (measured) *measured = err;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_choice[key] = {*moduli, err};
  }
  b200_tune_save_env();
  return B200_OK;
}

// Tuned-table lines for the choices: "ozaki2 <fp64> <k bucket> <target
// bits, hex> <moduli> <measured error>".
void b200_ozaki2_table_lines(std::string *text) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (const auto &kv : g_choice) {
    char line[128];
    snprintf(line, sizeof line, "ozaki2 %d %d %llx %d %.17g\n", std::get<0>(kv.first),
             std::get<1>(kv.first), std::get<2>(kv.first), kv.second.first, kv.second.second);
    *text += line;
  }
}

bool b200_ozaki2_table_parse(const char *line) {
  int fp64, kb, n;
  unsigned long long tb;
  double err;
  if (sscanf(line, "ozaki2 %d %d %llx %d %lg", &fp64, &kb, &tb, &n, &err) != 5) return false;
  if (fp64 < 0 || fp64 > 1 || kb < 0 || kb > 62 || n < 6 || n > B200_MAX_MODULI) return false;
  std::lock_guard<std::mutex> lk(g_mu);
  g_choice[std::make_tuple(fp64, kb, tb)] = {n, err};
  return true;
}

void b200_ozaki2_table_reset() {
  std::lock_guard<std::mutex> lk(g_mu);
  g_choice.clear();
}

extern "C" int mublis_b200_ozaki2_autotune(char dtype, mublis_trans_t trans_a, mublis_trans_t trans_b,
                                           int m, int n, int k, const void *a, int rs_a, int cs_a,
                                           const void *b, int rs_b, int cs_b, double target_err,
                                           int *moduli, double *measured_err) {
  B200_TRY(b200_init());
  if (dtype != 's' && dtype != 'd') return b200_set_error(B200_EINVAL, "ozaki2 tune: dtype");
  if (m <= 0 || n <= 0 || k <= 0) return b200_set_error(B200_EINVAL, "ozaki2 tune: empty problem");
  if (!moduli) return b200_set_error(B200_EINVAL, "ozaki2 tune: moduli is NULL");
  if (!b200_is_device_ptr(a) || !b200_is_device_ptr(b))
    return b200_set_error(B200_EINVAL, "ozaki2 tune: A and B must be device pointers");
  b200_l3_desc_t d;
  memset(&d, 0, sizeof d);
  d.dtype = dtype == 'd' ? B200_F64 : B200_F32;
  d.m = m;
  d.n = n;
  d.k = k;
  d.alpha = 1.0;
  d.npairs = 1;
  // op() as a stride swap (frame/l3/gemm.c:14-24).
  d.a[0] = a;
  d.rs_a[0] = trans_a == MUBLIS_TRANSPOSE ? cs_a : rs_a;
  d.cs_a[0] = trans_a == MUBLIS_TRANSPOSE ? rs_a : cs_a;
  d.b[0] = b;
  d.rs_b[0] = trans_b == MUBLIS_TRANSPOSE ? cs_b : rs_b;
  d.cs_b[0] = trans_b == MUBLIS_TRANSPOSE ? rs_b : cs_b;
  mublis_l3_operand_t gen = {MUBLIS_STRUC_GENERAL, MUBLIS_DENSE, MUBLIS_PACKM_DIAG_NONUNIT};
  d.product.domain.jp = d.product.domain.ji = d.product.domain.pi = MUBLIS_L3_ALL;
  d.product.a = gen;
  d.product.b = gen;
  d.form = B200_FORM_OZAKI2;
  B200_TRY(b200_ozaki2_choice(&d, target_err, moduli, measured_err, 1));
  return b200_stream_sync();
}
