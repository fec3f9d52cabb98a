// grouped.cu -- many independent GEMMs / left TRSMs of uneven sizes in one
// persistent launch each, plus the plan object that autotunes the tile shape
// and captures the launches in a CUDA graph for replay.
//
// The reference has no batched interface: every call runs the full driver
// (frame/l3/l3_driver.c) on one host thread.  For many small calls the B200
// cost is launch latency and packing passes, not flops, so the grouped path
// (a) reads operands directly from caller memory with bounds checks (no
// pack pass), (b) maps every output tile of every problem into one global
// tile index space (prefix sums over per-problem tile counts) walked by a
// persistent grid, and (c) solves each TRSM instance's column slab entirely
// on one CTA.
#include <algorithm>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "../../include/mublis_b200.h"
#include "tc_gemm.cuh"

namespace {

struct GemmEntry {
  long m, n, k;
  double alpha, beta;
  const void *a;
  long rs_a, cs_a;  // element (i, p) of op(A) at a[i*rs_a + p*cs_a]
  const void *b;
  long rs_b, cs_b;  // element (p, j) of op(B) at b[p*rs_b + j*cs_b]
  void *c;
  long rs_c, cs_c;  // element (i, j) of C at c[i*rs_c + j*cs_c]
  int tile0;        // first global tile index of this problem
  int tiles_m;
};

// ---- grouped GEMM kernel --------------------------------------------------------
//
// 256 threads as a 16 x 16 grid; each thread a TM x TN register tile, so a CTA
// covers (16*TM) x (16*TN).  Double-buffered shared memory with register
// prefetch of the next k-block; loads follow whichever operand stride is 1.

// Copies a run of V elements from shared memory (16- or 8-byte aligned when
// the run is that long) into registers with one vector load.
template <typename T, int V>
__device__ __forceinline__ void lds_run(T *dst, const T *src) {
  if constexpr (V * sizeof(T) == 16) {
    const uint4 x = *reinterpret_cast<const uint4 *>(src);
    memcpy(dst, &x, 16);
  } else if constexpr (V * sizeof(T) == 8) {
    const uint2 x = *reinterpret_cast<const uint2 *>(src);
    memcpy(dst, &x, 8);
  } else {
#pragma unroll
    for (int v = 0; v < V; ++v) dst[v] = src[v];
  }
}

// `table` may be null: then the single problem `one` (passed by value in the
// launch parameters) is the whole group -- the direct path for one small GEMM,
// with no table upload.
template <typename T, int TM, int TN>
__global__ void __launch_bounds__(256) grouped_gemm_kernel(const GemmEntry *__restrict__ table,
                                                           int nprob, int total_tiles,
                                                           const __grid_constant__ GemmEntry one) {
  constexpr int BM = 16 * TM, BN = 16 * TN, BK = sizeof(T) == 8 ? 8 : 16;
  constexpr int A_PER = BM * BK / 256, B_PER = BK * BN / 256;
  __shared__ __align__(16) T As[2][BK][BM];
  __shared__ __align__(16) T Bs[2][BK][BN];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  // Thread (tx, ty) holds rows row0 + (i % VM) + 16 VM (i / VM) and columns
  // col0 + (j % VN) + 16 VN (j / VN): runs of up to 16 bytes, so each k step
  // reads its A and B fragments with vector shared loads (one 16-byte load
  // per four floats instead of four 4-byte loads).
  constexpr int VM = TM * sizeof(T) >= 16 ? 16 / (int)sizeof(T) : TM;
  constexpr int VN = TN * sizeof(T) >= 16 ? 16 / (int)sizeof(T) : TN;
  const int row0 = ty * VM, col0 = tx * VN;

  // The table is followed by one int per output tile: the tile's problem.
  const int *tile_prob = table ? reinterpret_cast<const int *>(table + nprob) : nullptr;
  for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
    const GemmEntry &e = table ? table[tile_prob[tile]] : one;
    const int local = tile - e.tile0;
    const long m0 = (long)(local % e.tiles_m) * BM, n0 = (long)(local / e.tiles_m) * BN;
    const T *A = (const T *)e.a, *B = (const T *)e.b;
    const bool a_mfast = e.rs_a <= e.cs_a;  // i contiguous in memory
    const bool b_kfast = e.rs_b <= e.cs_b;  // p contiguous in memory

    T ra[A_PER], rb[B_PER];
    auto gload = [&](long k0) {
#pragma unroll
      for (int q = 0; q < A_PER; ++q) {
        int idx = tid + 256 * q;
        int i = a_mfast ? idx % BM : idx / BK, p = a_mfast ? idx / BM : idx % BK;
        long gi = m0 + i, gp = k0 + p;
        ra[q] = (gi < e.m && gp < e.k) ? A[gi * e.rs_a + gp * e.cs_a] : T(0);
      }
#pragma unroll
      for (int q = 0; q < B_PER; ++q) {
        int idx = tid + 256 * q;
        int p = b_kfast ? idx % BK : idx / BN, j = b_kfast ? idx / BK : idx % BN;
        long gp = k0 + p, gj = n0 + j;
        rb[q] = (gp < e.k && gj < e.n) ? B[gp * e.rs_b + gj * e.cs_b] : T(0);
      }
    };
    auto sstore = [&](int buf) {
#pragma unroll
      for (int q = 0; q < A_PER; ++q) {
        int idx = tid + 256 * q;
        int i = a_mfast ? idx % BM : idx / BK, p = a_mfast ? idx / BM : idx % BK;
        As[buf][p][i] = ra[q];
      }
#pragma unroll
      for (int q = 0; q < B_PER; ++q) {
        int idx = tid + 256 * q;
        int p = b_kfast ? idx % BK : idx / BN, j = b_kfast ? idx / BK : idx % BN;
        Bs[buf][p][j] = rb[q];
      }
    };

    // FP32 accumulates column pairs with the packed sm_100 FMA (__ffma2_rn:
    // two correctly rounded fmaf per instruction), halving the FMA issue
    // slots; each element's result is that of fmaf.
    constexpr bool PAIR = sizeof(T) == 4;
    constexpr int TNP = PAIR ? TN / 2 : TN;
    using Acc = typename std::conditional<PAIR, float2, T>::type;
    Acc acc[TM][TNP];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TNP; ++j) {
        if constexpr (PAIR) acc[i][j] = make_float2(0.f, 0.f);
        else acc[i][j] = T(0);
      }

    const int kblocks = (int)((e.k + BK - 1) / BK);
    __syncthreads();  // previous tile's readers are done with the buffers
    if (kblocks > 0) {
      gload(0);
      sstore(0);
    }
    __syncthreads();
    for (int kb = 0; kb < kblocks; ++kb) {
      const int cur = kb & 1;
      if (kb + 1 < kblocks) gload((long)(kb + 1) * BK);
#pragma unroll
      for (int p = 0; p < BK; ++p) {
        T af[TM], bf[TN];
#pragma unroll
        for (int g = 0; g < TM / VM; ++g) lds_run<T, VM>(af + g * VM, &As[cur][p][row0 + 16 * VM * g]);
#pragma unroll
        for (int g = 0; g < TN / VN; ++g) lds_run<T, VN>(bf + g * VN, &Bs[cur][p][col0 + 16 * VN * g]);
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TNP; ++j) {
            if constexpr (PAIR)
              acc[i][j] = __ffma2_rn(make_float2(af[i], af[i]),
                                     make_float2(bf[2 * j], bf[2 * j + 1]), acc[i][j]);
            else
              acc[i][j] = fma(af[i], bf[j], acc[i][j]);
          }
      }
      if (kb + 1 < kblocks) sstore(cur ^ 1);
      __syncthreads();
    }

    // Per row, the TN loads of C are issued before its stores (one memory
    // round trip per row rather than per element; small problems spend a
    // large share of their time here).  The FP64 8 x 8 variant, already at
    // 255 registers, keeps one element at a time.
    constexpr bool ROW_BATCH = !(sizeof(T) == 8 && TM * TN >= 64);
    const T alpha = (T)e.alpha, beta = (T)e.beta;
    T *Cm = (T *)e.c;
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const long gi = m0 + row0 + i % VM + 16 * VM * (i / VM);
      if (gi >= e.m) continue;
      T cv[TN];
      if constexpr (ROW_BATCH) {
#pragma unroll
        for (int j = 0; j < TN; ++j) {
          const long gj = n0 + col0 + j % VN + 16 * VN * (j / VN);
          cv[j] = gj < e.n && beta != T(0) ? Cm[gi * e.rs_c + gj * e.cs_c] : T(0);
        }
      }
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        const long gj = n0 + col0 + j % VN + 16 * VN * (j / VN);
        if (gj >= e.n) continue;
        T *cij = Cm + gi * e.rs_c + gj * e.cs_c;
        T aij;
        if constexpr (PAIR) aij = (j & 1) ? acc[i][j >> 1].y : acc[i][j >> 1].x;
        else aij = acc[i][j];
        T v = alpha * aij;
        if (beta != T(0)) v = fma(beta, ROW_BATCH ? cv[j] : *cij, v);
        *cij = v;
      }
    }
  }
}

// ---- grouped TRSM kernel ----------------------------------------------------------
//
// One CTA per (problem, 32-column slab of B): the slab (order <= 256 rows)
// lives in shared memory; the diagonal is walked in 32-row blocks: warp 0
// solves the block (reciprocal diagonal, multiplied), then all 8 warps
// update the rows below (lower) or above (upper) with the solved block.

struct TrsmEntry {
  long m, n;           // order and right-hand-side count
  double alpha;
  const void *a;
  long rs_a, cs_a;     // op(A) element (i, p) at a[i*rs_a + p*cs_a]
  void *b;
  long rs_b, cs_b;     // element (i, j) of B at b[i*rs_b + j*cs_b]
  int lower, unit;
  int slab0;           // first global slab index
};

constexpr int TRSM_MAX_ORDER = 256;
constexpr int TRSM_SLAB = 32;

template <typename T>
__global__ void __launch_bounds__(256) grouped_trsm_kernel(const TrsmEntry *__restrict__ table,
                                                           int nprob, int total_slabs) {
  extern __shared__ __align__(16) unsigned char trsm_smem[];
  T(*X)[TRSM_SLAB + 1] = reinterpret_cast<T(*)[TRSM_SLAB + 1]>(trsm_smem);
  T(*L)[33] = reinterpret_cast<T(*)[33]>(trsm_smem + sizeof(T) * TRSM_MAX_ORDER * (TRSM_SLAB + 1));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // The table is followed by one int per slab: the slab's problem.
  const int *slab_prob = reinterpret_cast<const int *>(table + nprob);
  for (int slab = blockIdx.x; slab < total_slabs; slab += gridDim.x) {
    const TrsmEntry &e = table[slab_prob[slab]];
    const long j0 = (long)(slab - e.slab0) * TRSM_SLAB;
    const int ncol = (int)min((long)TRSM_SLAB, e.n - j0);
    const int m = (int)e.m;
    const T *A = (const T *)e.a;
    T *Bm = (T *)e.b;
    const T alpha = (T)e.alpha;
    __syncthreads();
    for (int idx = tid; idx < m * TRSM_SLAB; idx += 256) {
      int i = idx % m, j = idx / m;
      X[i][j] = j < ncol ? alpha * Bm[i * e.rs_b + (j0 + j) * e.cs_b] : T(0);
    }
    __syncthreads();
    const int nblk = (m + 31) / 32;
    for (int q = 0; q < nblk; ++q) {
      const int b = e.lower ? q : nblk - 1 - q;
      const int r0 = b * 32, rb = min(32, m - r0);
      // diagonal block with reciprocal diagonal; the unstored triangle and a
      // unit diagonal are never read
      for (int idx = tid; idx < 32 * 32; idx += 256) {
        int i = idx % 32, p = idx / 32;
        T v = T(0);
        if (i < rb && p < rb) {
          if (i == p) v = e.unit ? T(1) : T(1) / A[(r0 + i) * e.rs_a + (r0 + i) * e.cs_a];
          else if (e.lower ? p < i : p > i) v = A[(r0 + i) * e.rs_a + (r0 + p) * e.cs_a];
        }
        L[i][p] = v;
      }
      __syncthreads();
      if (warp == 0) {  // lane = column of the slab
        if (e.lower) {
          for (int i = 0; i < rb; ++i) {
            T r = X[r0 + i][lane];
            for (int p = 0; p < i; ++p) r = fma(-L[i][p], X[r0 + p][lane], r);
            X[r0 + i][lane] = r * L[i][i];
          }
        } else {
          for (int i = rb - 1; i >= 0; --i) {
            T r = X[r0 + i][lane];
            for (int p = i + 1; p < rb; ++p) r = fma(-L[i][p], X[r0 + p][lane], r);
            X[r0 + i][lane] = r * L[i][i];
          }
        }
      }
      __syncthreads();
      // rows still to solve: below the block (lower) or above it (upper)
      const int u0 = e.lower ? r0 + rb : 0, u1 = e.lower ? m : r0;
      for (int idx = tid; idx < (u1 - u0) * TRSM_SLAB; idx += 256) {
        int i = u0 + idx / TRSM_SLAB, j = idx % TRSM_SLAB;
        T s = X[i][j];
        for (int p = 0; p < rb; ++p) s = fma(-A[i * e.rs_a + (r0 + p) * e.cs_a], X[r0 + p][j], s);
        X[i][j] = s;
      }
      __syncthreads();
    }
    for (int idx = tid; idx < m * TRSM_SLAB; idx += 256) {
      int i = idx % m, j = idx / m;
      if (j < ncol) Bm[i * e.rs_b + (j0 + j) * e.cs_b] = X[i][j];
    }
  }
}

// ---- host side ------------------------------------------------------------------

enum { TILE_32 = 0, TILE_64 = 1, TILE_128x64 = 2, TILE_128 = 3, TILE_VARIANTS = 4 };
const int kTileBM[TILE_VARIANTS] = {32, 64, 128, 128};
const int kTileBN[TILE_VARIANTS] = {32, 64, 64, 128};

int sm_count() { return b200_sm_count(); }

template <typename T>
int launch_gemm_variant(int variant, const GemmEntry *dtable, int nprob, int tiles,
                        cudaStream_t s, const GemmEntry *one = nullptr) {
  if (tiles <= 0) return B200_OK;
  const int grid = std::min(tiles, sm_count() * 4);
  GemmEntry single;
  if (one) single = *one; else memset(&single, 0, sizeof single);
  B200ProfScope prof(one ? (sizeof(T) == 4 ? "direct_sgemm" : "direct_dgemm")
                         : (sizeof(T) == 4 ? "grouped_sgemm" : "grouped_dgemm"), s);
  switch (variant) {
  case TILE_32: grouped_gemm_kernel<T, 2, 2><<<grid, 256, 0, s>>>(dtable, nprob, tiles, single); break;
  case TILE_64: grouped_gemm_kernel<T, 4, 4><<<grid, 256, 0, s>>>(dtable, nprob, tiles, single); break;
  case TILE_128x64: grouped_gemm_kernel<T, 8, 4><<<grid, 256, 0, s>>>(dtable, nprob, tiles, single); break;
  default: grouped_gemm_kernel<T, 8, 8><<<grid, 256, 0, s>>>(dtable, nprob, tiles, single); break;
  }
  B200_LAUNCH_CHECK();
  return B200_OK;
}

// Size classes the autotuner chooses a tile shape for (by max(m, n)).
int size_class(long m, long n) {
  long x = std::max(m, n);
  return x <= 48 ? 0 : (x <= 160 ? 1 : 2);
}
constexpr int NCLASS = 3;

struct GemmGroup {
  std::vector<GemmEntry> entries;  // host copy, tile0/tiles_m filled for `variant`
  GemmEntry *dtable = nullptr;     // entries, then the tile -> problem map
  size_t bytes = 0;                // allocated at dtable
  int tiles = 0;
  int variant = TILE_64;
};

// Host image of a class's device table for tile variant v: the entries
// (tile0 / tiles_m filled) followed by one int per output tile, the index
// of the tile's problem, so that a CTA finds its tile's problem with one
// load (a binary search over tile0 was a chain of ~12 dependent loads per
// tile).
std::vector<char> table_image(std::vector<GemmEntry> &es, int v, int &tiles) {
  int t = 0;
  for (auto &e : es) {
    e.tile0 = t;
    e.tiles_m = (int)b200_ceil_div(e.m, kTileBM[v]);
    t += e.tiles_m * (int)b200_ceil_div(e.n, kTileBN[v]);
  }
  tiles = t;
  const size_t head = sizeof(GemmEntry) * es.size();
  std::vector<char> img(head + sizeof(int) * (size_t)t);
  if (!es.empty()) memcpy(img.data(), es.data(), head);
  int *map = reinterpret_cast<int *>(img.data() + head);
  for (size_t q = 0; q < es.size(); ++q) {
    const int end = q + 1 < es.size() ? es[q + 1].tile0 : t;
    for (int x = es[q].tile0; x < end; ++x) map[x] = (int)q;
  }
  return img;
}

// Builds the device table of one class for a tile variant.
int build_group(std::vector<GemmEntry> &src, int variant, GemmGroup &g, cudaStream_t s) {
  g.entries = src;
  g.variant = variant;
  const std::vector<char> img = table_image(g.entries, variant, g.tiles);
  if (g.entries.empty()) return B200_OK;
  if (img.size() > g.bytes) {  // stream-ordered: earlier launches keep the old table
    b200_free(g.dtable);
    g.dtable = nullptr;
    g.bytes = 0;
    B200_TRY(b200_alloc((void **)&g.dtable, img.size()));
    g.bytes = img.size();
  }
  B200_CUDA_TRY(cudaMemcpyAsync(g.dtable, img.data(), img.size(), cudaMemcpyHostToDevice, s));
  return B200_OK;
}

int to_entries(char dtype, const mublis_b200_gemm_problem_t *p, int count,
               std::vector<GemmEntry> (&cls)[NCLASS]) {
  for (int q = 0; q < count; ++q) {
    const mublis_b200_gemm_problem_t &x = p[q];
    if (x.m < 0 || x.n < 0 || x.k < 0) return b200_set_error(B200_EINVAL, "grouped gemm: negative size");
    if (x.m == 0 || x.n == 0) continue;
    if (x.ldc < std::max(1, x.m)) return b200_set_error(B200_EINVAL, "grouped gemm: ldc too small");
    const bool upd = x.alpha != 0.0 && x.k > 0;
    if (!b200_is_device_ptr(x.c) || (upd && (!b200_is_device_ptr(x.a) || !b200_is_device_ptr(x.b))))
      return b200_set_error(B200_EINVAL, "grouped gemm: operands must be device pointers");
    GemmEntry e;
    memset(&e, 0, sizeof e);
    e.m = x.m;
    e.n = x.n;
    e.k = upd ? x.k : 0;  // alpha == 0: beta * C only, A and B never read
    e.alpha = x.alpha;
    e.beta = x.beta;
    e.a = x.a;
    e.b = x.b;
    e.rs_a = x.trans_a == MUBLIS_TRANSPOSE ? x.lda : 1;
    e.cs_a = x.trans_a == MUBLIS_TRANSPOSE ? 1 : x.lda;
    e.rs_b = x.trans_b == MUBLIS_TRANSPOSE ? x.ldb : 1;
    e.cs_b = x.trans_b == MUBLIS_TRANSPOSE ? 1 : x.ldb;
    e.c = x.c;
    e.rs_c = 1;
    e.cs_c = x.ldc;
    cls[size_class(x.m, x.n)].push_back(e);
  }
  (void)dtype;
  return B200_OK;
}

// Default tile per class, used until the autotuner has timed the classes.
const int kDefaultVariant[NCLASS] = {TILE_32, TILE_64, TILE_128};

template <typename T>
int run_groups(GemmGroup (&g)[NCLASS], cudaStream_t s) {
  for (int c = 0; c < NCLASS; ++c)
    if (g[c].tiles) B200_TRY(launch_gemm_variant<T>(g[c].variant, g[c].dtable, (int)g[c].entries.size(), g[c].tiles, s));
  return B200_OK;
}

// Autotuner: for each non-empty class time every tile variant on the
// class's actual problems (CUDA events, best of 2 after a warm-up) and keep
// the fastest.  Results are cached per (dtype, class, problem-count bucket)
// for the process.
std::mutex g_tune_mu;
int g_tuned[2][NCLASS][32];  // 0 = untuned, else variant + 1

// ---- tuned-table persistence ---------------------------------------------
//
// Text file: one key line, then one line per choice,
//   mublis_b200-tune <gpu name> sms=<n> cc=<major>.<minor> driver=<v> table=1
//   gemm <fp64 0/1> <size class> <count bucket> <tile variant>
// The key ties the file to a GPU model and driver (tile timings change with
// either); table=1 names this library's classes and variants.

constexpr int kTuneTable = 1;

std::string tune_key() {
  int dev = 0, drv = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return std::string();
  cudaDriverGetVersion(&drv);
  std::string name(prop.name);
  for (char &ch : name)
    if (ch == ' ' || ch == '\t') ch = '_';
  char buf[512];
  snprintf(buf, sizeof buf, "mublis_b200-tune %s sms=%d cc=%d.%d driver=%d table=%d",
           name.c_str(), prop.multiProcessorCount, prop.major, prop.minor, drv, kTuneTable);
  return buf;
}

int tune_save(const char *path) {
  if (!path || !*path) return b200_set_error(B200_EINVAL, "tune: empty path");
  const std::string key = tune_key();
  if (key.empty()) return b200_set_error(B200_ECUDA, "tune: no device to key the table to");
  std::string text = key + "\n";
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (int dt = 0; dt < 2; ++dt)
      for (int c = 0; c < NCLASS; ++c)
        for (int b = 0; b < 32; ++b)
          if (g_tuned[dt][c][b]) {
            char line[64];
            snprintf(line, sizeof line, "gemm %d %d %d %d\n", dt, c, b, g_tuned[dt][c][b] - 1);
            text += line;
          }
  }
  b200_ozaki2_table_lines(&text);
  const std::string tmp = std::string(path) + ".tmp";
  FILE *f = fopen(tmp.c_str(), "w");
  if (!f) return b200_set_error(B200_EINVAL, "tune: cannot write the table file");
  const bool ok = fwrite(text.data(), 1, text.size(), f) == text.size();
  if (fclose(f) != 0 || !ok || rename(tmp.c_str(), path) != 0) {
    remove(tmp.c_str());
    return b200_set_error(B200_EINVAL, "tune: cannot write the table file");
  }
  return B200_OK;
}

int tune_load(const char *path, int *entries) {
  if (entries) *entries = 0;
  if (!path || !*path) return b200_set_error(B200_EINVAL, "tune: empty path");
  FILE *f = fopen(path, "r");
  if (!f) return B200_OK;  // no table yet
  const std::string key = tune_key();
  char line[512];
  int loaded = 0;
  if (!key.empty() && fgets(line, sizeof line, f)) {
    line[strcspn(line, "\r\n")] = 0;
    if (key == line) {
      while (fgets(line, sizeof line, f)) {
        if (!strncmp(line, "ozaki2 ", 7)) {
          if (b200_ozaki2_table_parse(line)) ++loaded;
          continue;
        }
        int dt, c, b, v;
        if (sscanf(line, "gemm %d %d %d %d", &dt, &c, &b, &v) != 4) continue;
        if (dt < 0 || dt > 1 || c < 0 || c >= NCLASS || b < 0 || b >= 32 || v < 0 ||
            v >= TILE_VARIANTS)
          continue;
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[dt][c][b] = v + 1;
        ++loaded;
      }
    }
  }
  fclose(f);
  if (entries) *entries = loaded;
  return B200_OK;
}

const char *tune_env_path() {
  const char *p = getenv("MUBLIS_B200_TUNE_FILE");
  return p && *p ? p : nullptr;
}

void b200_tune_autosave() {
  if (const char *p = tune_env_path()) tune_save(p);  // best effort: tuning goes on regardless
}

template <typename T>
int autotune(std::vector<GemmEntry> (&cls)[NCLASS], GemmGroup (&g)[NCLASS], cudaStream_t s) {
  const int dt = sizeof(T) == 8;
  cudaEvent_t e0, e1;
  B200_CUDA_TRY(cudaEventCreate(&e0));
  B200_CUDA_TRY(cudaEventCreate(&e1));
  for (int c = 0; c < NCLASS; ++c) {
    if (cls[c].empty()) continue;
    int bucket = 31 - __builtin_clz((unsigned)cls[c].size());
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      if (g_tuned[dt][c][bucket]) {
        B200_TRY(build_group(cls[c], g_tuned[dt][c][bucket] - 1, g[c], s));
        continue;
      }
    }
    float best = 1e30f;
    int best_v = kDefaultVariant[c];
    for (int v = 0; v < TILE_VARIANTS; ++v) {
      B200_TRY(build_group(cls[c], v, g[c], s));
      float ms_best = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {
        B200_CUDA_TRY(cudaEventRecord(e0, s));
        B200_TRY(launch_gemm_variant<T>(v, g[c].dtable, (int)g[c].entries.size(), g[c].tiles, s));
        B200_CUDA_TRY(cudaEventRecord(e1, s));
        B200_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) ms_best = std::min(ms_best, ms);
      }
      if (ms_best < best) { best = ms_best; best_v = v; }
    }
    B200_TRY(build_group(cls[c], best_v, g[c], s));
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tuned[dt][c][bucket] = best_v + 1;
    }
    b200_tune_autosave();
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return B200_OK;
}

// Note: the autotuner's trial launches write C (they are real executions of
// the grouped product); a plan therefore snapshots and restores every C
// before tuning.  See plan_gemm below.

struct TrsmGroup {
  std::vector<TrsmEntry> entries;
  TrsmEntry *dtable = nullptr;  // entries, then the slab -> problem map
  int slabs = 0;
  std::vector<int> fallback;  // problems too large for the one-CTA solve
};

// Host image of a TRSM group's device table: the entries followed by one
// int per 32-column slab, the index of the slab's problem.
std::vector<char> trsm_table_image(const TrsmGroup &g) {
  const size_t head = sizeof(TrsmEntry) * g.entries.size();
  std::vector<char> img(head + sizeof(int) * (size_t)g.slabs);
  if (!g.entries.empty()) memcpy(img.data(), g.entries.data(), head);
  int *map = reinterpret_cast<int *>(img.data() + head);
  for (size_t q = 0; q < g.entries.size(); ++q) {
    const int end = q + 1 < g.entries.size() ? g.entries[q + 1].slab0 : g.slabs;
    for (int x = g.entries[q].slab0; x < end; ++x) map[x] = (int)q;
  }
  return img;
}

int to_trsm(const mublis_b200_trsm_problem_t *p, int count, TrsmGroup &g, cudaStream_t s) {
  int slabs = 0;
  for (int q = 0; q < count; ++q) {
    const mublis_b200_trsm_problem_t &x = p[q];
    if (x.m < 0 || x.n < 0) return b200_set_error(B200_EINVAL, "grouped trsm: negative size");
    if (x.m == 0 || x.n == 0) continue;
    if (x.uplo != MUBLIS_LOWER && x.uplo != MUBLIS_UPPER)
      return b200_set_error(B200_EINVAL, "grouped trsm: uplo must be lower or upper");
    if (!b200_is_device_ptr(x.b) || (x.alpha != 0.0 && !b200_is_device_ptr(x.a)))
      return b200_set_error(B200_EINVAL, "grouped trsm: operands must be device pointers");
    if (x.m > TRSM_MAX_ORDER || x.alpha == 0.0) {
      g.fallback.push_back(q);
      continue;
    }
    TrsmEntry e;
    memset(&e, 0, sizeof e);
    e.m = x.m;
    e.n = x.n;
    e.alpha = x.alpha;
    e.a = x.a;
    // trans folds into strides and flips the triangle (frame/l3/trsm.c:49-54)
    const bool tr = x.trans_a == MUBLIS_TRANSPOSE;
    e.rs_a = tr ? x.lda : 1;
    e.cs_a = tr ? 1 : x.lda;
    e.lower = (x.uplo == MUBLIS_LOWER) != tr;
    e.unit = x.diag == MUBLIS_UNIT_DIAG;
    e.b = x.b;
    e.rs_b = 1;
    e.cs_b = x.ldb;
    e.slab0 = slabs;
    slabs += (int)b200_ceil_div(x.n, TRSM_SLAB);
    g.entries.push_back(e);
  }
  g.slabs = slabs;
  if (g.entries.empty()) return B200_OK;
  const std::vector<char> img = trsm_table_image(g);
  B200_TRY(b200_alloc((void **)&g.dtable, img.size()));
  B200_CUDA_TRY(cudaMemcpyAsync(g.dtable, img.data(), img.size(), cudaMemcpyHostToDevice, s));
  return B200_OK;
}

template <typename T>
int launch_trsm_group(TrsmGroup &g, cudaStream_t s) {
  if (g.slabs == 0) return B200_OK;
  const int grid = std::min(g.slabs, sm_count() * 4);
  const size_t smem = sizeof(T) * (TRSM_MAX_ORDER * (TRSM_SLAB + 1) + 32 * 33);
  static std::once_flag once;
  static int conf = B200_OK;
  B200_TRY(b200_once(once, conf, "grouped trsm: set-up failed", [&]() -> int {
    B200_CUDA_TRY(cudaFuncSetAttribute(grouped_trsm_kernel<T>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return B200_OK;
  }));
  B200ProfScope prof(sizeof(T) == 4 ? "grouped_strsm" : "grouped_dtrsm", s);
  grouped_trsm_kernel<T><<<grid, 256, smem, s>>>(g.dtable, (int)g.entries.size(), g.slabs);
  B200_LAUNCH_CHECK();
  return B200_OK;
}

int trsm_fallback(char dtype, const mublis_b200_trsm_problem_t *p, const std::vector<int> &idx) {
  for (int q : idx) {
    const mublis_b200_trsm_problem_t &x = p[q];
    int st = dtype == 'd'
                 ? mublis_dtrsm(MUBLIS_LEFT, (mublis_uplo_t)x.uplo, (mublis_trans_t)x.trans_a,
                                (mublis_diag_t)x.diag, x.m, x.n, x.alpha, (const double *)x.a, 1,
                                x.lda, (double *)x.b, 1, x.ldb)
                 : mublis_strsm(MUBLIS_LEFT, (mublis_uplo_t)x.uplo, (mublis_trans_t)x.trans_a,
                                (mublis_diag_t)x.diag, x.m, x.n, (float)x.alpha, (const float *)x.a,
                                1, x.lda, (float *)x.b, 1, x.ldb);
    if (st) return st;
  }
  return B200_OK;
}

}  // namespace

// ---- plans ------------------------------------------------------------------------

struct mublis_b200_plan {
  char dtype = 's';
  int kind = 0;  // 0 gemm, 1 trsm
  GemmGroup gg[NCLASS];
  TrsmGroup tg;
  b200_tcg *tcg = nullptr;  // FP32 GEMMs in the fp16x3 form
  std::vector<mublis_b200_trsm_problem_t> trsm_problems;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

template <typename T>
int plan_gemm(mublis_b200_plan *pl, const mublis_b200_gemm_problem_t *p, int count) {
  cudaStream_t s = b200_cur_stream();
  std::vector<GemmEntry> cls[NCLASS];
  B200_TRY(to_entries(pl->dtype, p, count, cls));
  // The tuner's trials are real executions; keep every C and put it back.
  std::vector<void *> saved(count, nullptr);
  for (int q = 0; q < count; ++q) {
    if (p[q].m == 0 || p[q].n == 0) continue;
    size_t bytes = (size_t)p[q].ldc * (p[q].n - 1) * sizeof(T) + (size_t)p[q].m * sizeof(T);
    B200_TRY(b200_alloc(&saved[q], bytes));
    B200_CUDA_TRY(cudaMemcpyAsync(saved[q], p[q].c, bytes, cudaMemcpyDeviceToDevice, s));
  }
  int st = autotune<T>(cls, pl->gg, s);
  for (int q = 0; q < count; ++q) {
    if (!saved[q]) continue;
    size_t bytes = (size_t)p[q].ldc * (p[q].n - 1) * sizeof(T) + (size_t)p[q].m * sizeof(T);
    if (cudaMemcpyAsync(p[q].c, saved[q], bytes, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      st = b200_set_error(B200_ECUDA, "plan: restoring C failed");
    b200_free(saved[q]);
  }
  return st;
}

// FP32 groups run in the fp16x3 tensor-core form (tc_grouped.cu) when that
// is the FP32 form; every other form runs the plain grouped kernel.
bool tc_grouped(char dtype) {
  return dtype == 's' && b200_get_default_form(B200_F32) == B200_FORM_FP16X3;
}

int capture(mublis_b200_plan *pl) {
  cudaStream_t s = b200_cur_stream();
  B200_TRY(b200_stream_sync());
  B200_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int st;
  if (pl->tcg)
    st = b200_tcg_run(pl->tcg, s);
  else if (pl->kind == 0)
    st = pl->dtype == 'd' ? run_groups<double>(pl->gg, s) : run_groups<float>(pl->gg, s);
  else
    st = pl->dtype == 'd' ? launch_trsm_group<double>(pl->tg, s) : launch_trsm_group<float>(pl->tg, s);
  cudaError_t e = cudaStreamEndCapture(s, &pl->graph);
  if (st != B200_OK) return st;
  B200_CUDA_TRY(e);
  B200_CUDA_TRY(cudaGraphInstantiate(&pl->exec, pl->graph, 0));
  return B200_OK;
}

}  // namespace

// ---- descriptor-based asynchronous entry points (the request server) --------

extern "C" int b200_l3_is_plain_gemm(const b200_l3_desc_t *d) {
  const mublis_l3_product_t &p = d->product;
  return d->npairs == 1 && p.domain.jp == MUBLIS_L3_ALL && p.domain.ji == MUBLIS_L3_ALL &&
         p.domain.pi == MUBLIS_L3_ALL && p.a.struc == MUBLIS_STRUC_GENERAL &&
         p.b.struc == MUBLIS_STRUC_GENERAL;
}

// Without a tuned choice: the class's default tile, stepped down to smaller
// tiles while the group would leave more than half of the SMs without a
// tile (a few 512 x 512 products, as TRSM's inverse doubling issues, are 16
// tiles each at 128 x 128).
int fill_variant(const std::vector<GemmEntry> &es, int v) {
  static const int smaller[TILE_VARIANTS] = {-1, TILE_32, TILE_64, TILE_128x64};
  auto tiles = [&](int var) {
    long t = 0;
    for (const auto &e : es)
      t += b200_ceil_div(e.m, kTileBM[var]) * b200_ceil_div(e.n, kTileBN[var]);
    return t;
  };
  while (smaller[v] >= 0 && 2 * tiles(v) < sm_count()) v = smaller[v];
  return v;
}

extern "C" int b200_grouped_gemm_async(int dtype, const b200_l3_desc_t *const *descs, int count,
                                       void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<GemmEntry> cls[NCLASS];
  for (int q = 0; q < count; ++q) {
    const b200_l3_desc_t &d = *descs[q];
    if (d.m <= 0 || d.n <= 0) continue;
    if (!b200_l3_is_plain_gemm(&d) || d.dtype != dtype)
      return b200_set_error(B200_EINVAL, "grouped: not a plain GEMM of this precision");
    GemmEntry e;
    memset(&e, 0, sizeof e);
    e.m = d.m;
    e.n = d.n;
    e.k = d.alpha != 0.0 ? d.k : 0;
    e.alpha = d.alpha;
    e.beta = d.beta;
    e.a = d.a[0];
    e.rs_a = d.rs_a[0];
    e.cs_a = d.cs_a[0];
    e.b = d.b[0];
    e.rs_b = d.rs_b[0];
    e.cs_b = d.cs_b[0];
    e.c = d.c;
    e.rs_c = d.rs_c;
    e.cs_c = d.cs_c;
    cls[size_class(d.m, d.n)].push_back(e);
  }
  GemmGroup g[NCLASS];
  int st = B200_OK;
  for (int c = 0; c < NCLASS && st == B200_OK; ++c) {
    if (cls[c].empty()) continue;
    int bucket = 31 - __builtin_clz((unsigned)cls[c].size());
    int v;
    bool tuned;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      tuned = g_tuned[dtype == B200_F64][c][bucket] != 0;
      v = tuned ? g_tuned[dtype == B200_F64][c][bucket] - 1 : kDefaultVariant[c];
    }
    if (!tuned) v = fill_variant(cls[c], v);
    g[c].entries = cls[c];
    g[c].variant = v;
    const std::vector<char> img = table_image(g[c].entries, v, g[c].tiles);
    if (cudaMallocAsync((void **)&g[c].dtable, img.size(), s) != cudaSuccess ||
        cudaMemcpyAsync(g[c].dtable, img.data(), img.size(), cudaMemcpyHostToDevice, s) !=
            cudaSuccess)
      st = b200_set_error(B200_ECUDA, "grouped: table upload failed");
  }
  if (st == B200_OK)
    st = dtype == B200_F64 ? run_groups<double>(g, s) : run_groups<float>(g, s);
  for (auto &x : g)
    if (x.dtable) cudaFreeAsync(x.dtable, s);
  return st;
}

// One small plain GEMM without packing: the grouped kernel with the problem
// in its launch parameters (used by the TRSM recursion for thin updates).
extern "C" int b200_gemm_direct_min_rows(const b200_l3_desc_t *d, int min_rows);

extern "C" int b200_gemm_direct(const b200_l3_desc_t *d) { return b200_gemm_direct_min_rows(d, 0); }

// min_rows: smallest tile height allowed (an in-place product needs a tile
// to cover all rows of the block it overwrites).
extern "C" int b200_gemm_direct_min_rows(const b200_l3_desc_t *d, int min_rows) {
  if (d->m <= 0 || d->n <= 0) return B200_OK;
  if (!b200_l3_is_plain_gemm(d)) return b200_set_error(B200_EINVAL, "direct gemm: not plain");
  GemmEntry e;
  memset(&e, 0, sizeof e);
  e.m = d->m;
  e.n = d->n;
  e.k = d->alpha != 0.0 ? d->k : 0;
  e.alpha = d->alpha;
  e.beta = d->beta;
  e.a = d->a[0];
  e.rs_a = d->rs_a[0];
  e.cs_a = d->cs_a[0];
  e.b = d->b[0];
  e.rs_b = d->rs_b[0];
  e.cs_b = d->cs_b[0];
  e.c = d->c;
  e.rs_c = d->rs_c;
  e.cs_c = d->cs_c;
  int v = std::max(d->m, d->n) <= 64 ? TILE_32 : (std::min(d->m, d->n) <= 128 ? TILE_64 : TILE_128);
  while (kTileBM[v] < min_rows && v < TILE_128) ++v;
  if (kTileBM[v] < min_rows) return b200_set_error(B200_EINVAL, "direct gemm: tile too short");
  e.tile0 = 0;
  e.tiles_m = (int)b200_ceil_div(e.m, kTileBM[v]);
  const int tiles = e.tiles_m * (int)b200_ceil_div(e.n, kTileBN[v]);
  cudaStream_t s = b200_cur_stream();
  return d->dtype == B200_F64 ? launch_gemm_variant<double>(v, nullptr, 1, tiles, s, &e)
                              : launch_gemm_variant<float>(v, nullptr, 1, tiles, s, &e);
}

extern "C" int b200_grouped_trsm_async(int dtype, const b200_trsm_desc_t *const *descs, int count,
                                       void *stream) {
  cudaStream_t s = (cudaStream_t)stream;
  TrsmGroup g;
  int slabs = 0;
  for (int q = 0; q < count; ++q) {
    const b200_trsm_desc_t &d = *descs[q];
    if (d.m <= 0 || d.n <= 0) continue;
    if (d.m > TRSM_MAX_ORDER || d.dtype != dtype || d.alpha == 0.0)
      return b200_set_error(B200_EINVAL, "grouped: TRSM not batchable");
    TrsmEntry e;
    memset(&e, 0, sizeof e);
    e.m = d.m;
    e.n = d.n;
    e.alpha = d.alpha;
    e.a = d.a;
    e.rs_a = d.rs_a;
    e.cs_a = d.cs_a;
    e.lower = d.uplo == MUBLIS_LOWER;
    e.unit = d.unit_diag != 0;
    e.b = d.b;
    e.rs_b = d.rs_b;
    e.cs_b = d.cs_b;
    e.slab0 = slabs;
    slabs += (int)b200_ceil_div(d.n, TRSM_SLAB);
    g.entries.push_back(e);
  }
  g.slabs = slabs;
  if (g.entries.empty()) return B200_OK;
  const std::vector<char> img = trsm_table_image(g);
  if (cudaMallocAsync((void **)&g.dtable, img.size(), s) != cudaSuccess ||
      cudaMemcpyAsync(g.dtable, img.data(), img.size(), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return b200_set_error(B200_ECUDA, "grouped: table upload failed");
  int st = dtype == B200_F64 ? launch_trsm_group<double>(g, s) : launch_trsm_group<float>(g, s);
  cudaFreeAsync(g.dtable, s);
  return st;
}

extern "C" {

int mublis_b200_gemm_grouped(char dtype, const mublis_b200_gemm_problem_t *problems, int count) {
  if (count < 0 || (count > 0 && !problems)) return b200_set_error(B200_EINVAL, "grouped gemm: bad arguments");
  if (dtype != 's' && dtype != 'd') return b200_set_error(B200_EINVAL, "grouped gemm: dtype is 's' or 'd'");
  if (count == 0) return B200_OK;
  B200_TRY(b200_init());
  cudaStream_t s = b200_cur_stream();
  if (tc_grouped(dtype)) {
    b200_tcg *g = nullptr;
    B200_TRY(b200_tcg_create(problems, count, &g));
    int st = b200_tcg_run(g, s);
    if (st == B200_OK) st = b200_stream_sync();
    b200_tcg_destroy(g);
    return st == B200_OK ? b200_stream_sync() : st;
  }
  std::vector<GemmEntry> cls[NCLASS];
  B200_TRY(to_entries(dtype, problems, count, cls));
  GemmGroup g[NCLASS];
  int st = B200_OK;
  for (int c = 0; c < NCLASS && st == B200_OK; ++c) {
    int bucket = cls[c].empty() ? 0 : 31 - __builtin_clz((unsigned)cls[c].size());
    int v;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      v = g_tuned[dtype == 'd'][c][bucket] ? g_tuned[dtype == 'd'][c][bucket] - 1 : kDefaultVariant[c];
    }
    st = build_group(cls[c], v, g[c], s);
  }
  if (st == B200_OK) st = dtype == 'd' ? run_groups<double>(g, s) : run_groups<float>(g, s);
  if (st == B200_OK) st = b200_stream_sync();
  for (auto &x : g) b200_free(x.dtable);
  return st == B200_OK ? b200_stream_sync() : st;
}

int mublis_b200_trsm_grouped(char dtype, const mublis_b200_trsm_problem_t *problems, int count) {
  if (count < 0 || (count > 0 && !problems)) return b200_set_error(B200_EINVAL, "grouped trsm: bad arguments");
  if (dtype != 's' && dtype != 'd') return b200_set_error(B200_EINVAL, "grouped trsm: dtype is 's' or 'd'");
  if (count == 0) return B200_OK;
  B200_TRY(b200_init());
  cudaStream_t s = b200_cur_stream();
  TrsmGroup g;
  int st = to_trsm(problems, count, g, s);
  if (st == B200_OK) st = dtype == 'd' ? launch_trsm_group<double>(g, s) : launch_trsm_group<float>(g, s);
  if (st == B200_OK) st = b200_stream_sync();
  b200_free(g.dtable);
  if (st == B200_OK) st = b200_stream_sync();
  if (st == B200_OK) st = trsm_fallback(dtype, problems, g.fallback);
  return st;
}

int mublis_b200_plan_gemm_grouped(char dtype, const mublis_b200_gemm_problem_t *problems,
                                  int count, mublis_b200_plan_t **plan) {
  if (!plan || count < 0 || (count > 0 && !problems) || (dtype != 's' && dtype != 'd'))
    return b200_set_error(B200_EINVAL, "plan: bad arguments");
  *plan = nullptr;
  B200_TRY(b200_init());
  auto *pl = new mublis_b200_plan;
  pl->dtype = dtype;
  pl->kind = 0;
  int st = tc_grouped(dtype) ? b200_tcg_create(problems, count, &pl->tcg)
           : dtype == 'd'    ? plan_gemm<double>(pl, problems, count)
                             : plan_gemm<float>(pl, problems, count);
  if (st == B200_OK) st = capture(pl);
  if (st != B200_OK) {
    mublis_b200_plan_destroy(pl);
    return st;
  }
  *plan = pl;
  return b200_stream_sync();
}

int mublis_b200_plan_trsm_grouped(char dtype, const mublis_b200_trsm_problem_t *problems,
                                  int count, mublis_b200_plan_t **plan) {
  if (!plan || count < 0 || (count > 0 && !problems) || (dtype != 's' && dtype != 'd'))
    return b200_set_error(B200_EINVAL, "plan: bad arguments");
  *plan = nullptr;
  B200_TRY(b200_init());
  auto *pl = new mublis_b200_plan;
  pl->dtype = dtype;
  pl->kind = 1;
  int st = to_trsm(problems, count, pl->tg, b200_cur_stream());
  if (st == B200_OK && !pl->tg.fallback.empty())
    st = b200_set_error(B200_EINVAL, "plan: every TRSM must have order <= 256 and alpha != 0");
  if (st == B200_OK) st = capture(pl);
  if (st != B200_OK) {
    mublis_b200_plan_destroy(pl);
    return st;
  }
  *plan = pl;
  return b200_stream_sync();
}

int mublis_b200_plan_run(mublis_b200_plan_t *plan) {
  if (!plan || !plan->exec) return b200_set_error(B200_EINVAL, "plan: not instantiated");
  cudaStream_t s = b200_cur_stream();
  {
    B200ProfScope prof("plan_graph", s);
    B200_CUDA_TRY(cudaGraphLaunch(plan->exec, s));
  }
  return b200_stream_sync();
}

int mublis_b200_plan_destroy(mublis_b200_plan_t *plan) {
  if (!plan) return B200_OK;
  if (plan->exec) cudaGraphExecDestroy(plan->exec);
  if (plan->graph) cudaGraphDestroy(plan->graph);
  for (auto &g : plan->gg) b200_free(g.dtable);
  b200_free(plan->tg.dtable);
  b200_tcg_destroy(plan->tcg);
  b200_stream_sync();
  delete plan;
  return B200_OK;
}

}  // extern "C"

// ---- tuned-table API (include/mublis_b200.h) ---------------------------------

extern "C" void b200_tune_autoload(void) {
  if (const char *p = tune_env_path()) tune_load(p, nullptr);
}

extern "C" int mublis_b200_tune_save(const char *path) {
  B200_TRY(b200_init());
  return tune_save(path);
}

extern "C" int mublis_b200_tune_load(const char *path, int *entries) {
  if (entries) *entries = 0;
  B200_TRY(b200_init());
  return tune_load(path, entries);
}

void b200_tune_save_env() { b200_tune_autosave(); }

extern "C" int mublis_b200_tune_reset(void) {
  b200_ozaki2_table_reset();
  std::lock_guard<std::mutex> lk(g_tune_mu);
  memset(g_tuned, 0, sizeof g_tuned);
  return B200_OK;
}
