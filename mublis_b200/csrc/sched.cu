// sched.cu -- the device tile scheduler's host half: which output tiles a
// product writes, how heavy each is, and how many k-chunks (split-K) each
// tile is cut into for the persistent GEMM kernels.
//
// The reference's five-loop driver walks nc / mc / kc blocks in a fixed
// order on one thread (frame/l3/l3_driver.c:126-239), skipping blocks
// outside the written triangle (:145-147,165-171) and clipping each block's
// k range to the product's support (:130,148-150,163,171).  On the B200 the
// output tiles are the unit of parallel work: persistent CTAs (one or two
// per SM) take (tile, k-chunk) units from a device counter, heaviest tile
// first, and a tile cut into S chunks is finished by the last chunk to
// arrive, which adds the chunks' sums in chunk order.  S is chosen here from
// a list-scheduling simulation of exactly that, so that a call whose tile
// count leaves the last wave part-empty (1024 tiles on 296 CTAs), or that
// has few tiles and a long k (SYRK with n = 1024, k = 8192: 36 tiles), keeps
// every SM busy.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <queue>
#include <tuple>
#include <vector>

#include "kernels.cuh"

void b200_tile_list(long m, long n, long k, int BM, int BN, int BK, b200_tile_domain_t dom,
                    std::vector<int2> *list, std::vector<int> *costs) {
  const long tiles_m = b200_ceil_div(m, BM), tiles_n = b200_ceil_div(n, BN);
  std::vector<std::pair<int, int2>> tl;
  for (long tm = 0; tm < tiles_m; ++tm)
    for (long tn = 0; tn < tiles_n; ++tn) {
      const long m0 = tm * BM, n0 = tn * BN;
      if (dom.ji == MUBLIS_L3_LOWER && n0 >= m0 + BM) continue;
      if (dom.ji == MUBLIS_L3_UPPER && n0 + BN <= m0) continue;
      long kb = 0, ke = k;
      if (dom.jp == MUBLIS_L3_LOWER) kb = std::max(kb, n0);       // j <= p
      if (dom.jp == MUBLIS_L3_UPPER) ke = std::min(ke, n0 + BN);  // j >= p
      if (dom.pi == MUBLIS_L3_LOWER) ke = std::min(ke, m0 + BM);  // p <= i
      if (dom.pi == MUBLIS_L3_UPPER) kb = std::max(kb, m0);       // p >= i
      const long cost = ke > kb ? (ke + BK - 1) / BK - kb / BK : 0;
      tl.push_back({(int)cost, make_int2((int)tm, (int)tn)});
    }
  std::stable_sort(tl.begin(), tl.end(), [](const std::pair<int, int2> &x,
                                            const std::pair<int, int2> &y) {
    return x.first > y.first;
  });
  if (list) {
    list->resize(tl.size());
    for (size_t i = 0; i < tl.size(); ++i) (*list)[i] = tl[i].second;
  }
  if (costs) {
    costs->resize(tl.size());
    for (size_t i = 0; i < tl.size(); ++i) (*costs)[i] = tl[i].first;
  }
}

namespace {

// Per-unit cost beyond its k-blocks, in k-block times: fetching the unit,
// filling the copy pipeline and the epilogue.  A split unit also stores its
// partial sums and the tile's last one reloads them all, and concurrent
// k-chunks of one tile share less of the operand panels in L2; the
// caller's split_cost covers that.  Measured on B200: a split that the
// simulation credits with under 10% is slower in practice (SGEMM 4096^3
// on 296 CTAs: S = 2 modelled 9% faster, measured 4.5% slower), while
// tile-starved calls gain severalfold (SYRK n = 1024, k = 8192: 36 tiles,
// FP32 10.9 -> 27.8 TF/s, FP64 7.2 -> 19.9), so S > 1 must beat S = 1 by
// 10% in the model.
constexpr double UNIT_COST = 1.5, SPLIT_GAIN = 0.9;
constexpr int MAX_SPLITS = 16, MIN_CHUNK = 8;
constexpr long MAX_SIM_UNITS = 1 << 16;

// Finish time of `units` (costs in order) list-scheduled on `slots` workers
// that each take the next unit when free.
double simulate(const std::vector<double> &units, long slots) {
  if ((long)units.size() <= slots) {
    double mx = 0;
    for (double c : units) mx = std::max(mx, c);
    return mx;
  }
  std::priority_queue<double, std::vector<double>, std::greater<double>> free_at;
  for (long i = 0; i < slots; ++i) free_at.push(0.0);
  double end = 0;
  for (double c : units) {
    const double t = free_at.top() + c;
    free_at.pop();
    free_at.push(t);
    end = std::max(end, t);
  }
  return end;
}

std::mutex g_mu;
std::map<std::tuple<long, long, long, int, int, int, int, int, int, long, double>, int> g_cache;

}  // namespace

int b200_split_for(long m_full, long n_full, long k, int BM, int BN, int BK,
                   b200_tile_domain_t dom, long slots, double split_cost) {
  if (m_full <= 0 || n_full <= 0 || k <= 0 || slots <= 0) return 1;
  // MUBLIS_B200_SPLIT=<S> fixes the split count (1: no split-K), for tuning.
  static const int forced = [] {
    const char *e = getenv("MUBLIS_B200_SPLIT");
    return e ? atoi(e) : 0;
  }();
  if (forced > 0) return std::min(forced, MAX_SPLITS);
  const auto key = std::make_tuple(m_full, n_full, k, BM, BN, BK, dom.jp, dom.ji, dom.pi, slots,
                                   split_cost);
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_cache.find(key);
    if (it != g_cache.end()) return it->second;
  }
  std::vector<int> costs;
  b200_tile_list(m_full, n_full, k, BM, BN, BK, dom, nullptr, &costs);
  const int heaviest = costs.empty() ? 0 : costs.front();
  int smax = std::min(MAX_SPLITS, std::max(1, heaviest / MIN_CHUNK));
  while (smax > 1 && (long)costs.size() * smax > MAX_SIM_UNITS) --smax;
  int best = 1;
  double best_t = 0, t1 = 0;
  std::vector<double> units;
  for (int S = 1; S <= smax; ++S) {
    units.clear();
    for (int c : costs) {
      const int per = (c + S - 1) / S;
      for (int q = 0; q < S; ++q) {
        const int len = std::max(0, std::min(per, c - q * per));
        units.push_back(len + UNIT_COST + (S > 1 ? split_cost : 0.0));
      }
    }
    const double t = simulate(units, slots);
    if (S == 1) {
      t1 = t;
      best_t = t;
    } else if (t < SPLIT_GAIN * t1 && t < best_t) {  // a split must win by 10%
      best = S;
      best_t = t;
    }
  }
  std::lock_guard<std::mutex> lk(g_mu);
  g_cache[key] = best;
  return best;
}
