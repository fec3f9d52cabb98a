// gemm_simt.cu -- plain FP32 / FP64 GEMM on the FMA pipes: the device
// form of the reference's five-loop driver (frame/l3/l3_driver.c:126-239)
// plus its micro-kernel (include/mublis_instantiate.h:37-52).
//
// One CTA per output tile (BM x BN), 256 threads, each thread an 8 x TN
// register tile laid out CUTLASS-SIMT style (4 x 8 threads per warp,
// 16-byte fragments spaced so that every shared-memory fragment load is a
// broadcast or a single 128-byte wavefront).  Operands come from packed MN-major panels (pack.cu)
// through a STAGES-deep cp.async pipeline; packing zero-pads every edge, so
// the main loop has no bounds checks.
//
// Domain handling replaces the reference's block pruning:
//   ji  -- tiles wholly outside the written triangle exit at once
//          (block_is_outside, l3_driver.c:145-147,165-171); partial tiles
//          are masked element-wise in the epilogue (:217-233);
//   jp, pi -- the tile's k-range is clipped to the product's support
//          (:130,148-150,163,171), e.g. TRMM does half the work of GEMM.
// Epilogue: C = alpha*acc + beta*C, and beta == 0 never reads C
// (:111-112, :224-225).  A tile with an empty k-range writes beta*C, which is
// the reference's "no update" pass (:88-121).
//
// Split-K (the reference's pc loop, l3_driver.c:126-135, spread over CTAs):
// a call with too few tiles to fill the GPU for its k (sched.cu decides,
// from the whole call's shape) runs on persistent CTAs that take (tile,
// k-chunk) units from a counter; each chunk stores its sums and the last
// chunk of a tile to finish adds them in chunk order and runs the epilogue,
// so the result does not depend on which CTA ran what.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "kernels.cuh"

namespace {

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// One 16-byte shared-memory fragment: 4 floats or 2 doubles.
__device__ __forceinline__ void lds16(float (&d)[4], const float *p) {
  float4 v = *reinterpret_cast<const float4 *>(p);
  d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
}
__device__ __forceinline__ void lds16(double (&d)[2], const double *p) {
  double2 v = *reinterpret_cast<const double2 *>(p);
  d[0] = v.x; d[1] = v.y;
}

// One output tile per CTA (block index -> tile, rasterised in groups of 8
// along M); tiles outside the written triangle exit at once.  Used for
// every call that is not split along k: a persistent schedule of the same
// tiles measured no faster (SGEMM 4096^3: 55.8 vs 55.6 TF/s), the tiles'
// own efficiency, not the last wave, being the limit there.
template <typename T, int BM, int BN, int BK, int WARPS_M, int WARPS_N, int STAGES, int MINB,
          bool PAIR = false>
__global__ void __launch_bounds__(256, MINB) simt_tile_kernel(SimtGemmArgs<T> p) {
  constexpr int NT = 256;
  constexpr int WTM = BM / WARPS_M, WTN = BN / WARPS_N;
  constexpr int TM = WTM / 4, TN = WTN / 8;
  // Fragments are 16-byte chunks of CW elements; a thread's chunks are
  // spaced so that one warp-wide load touches 4 (A) or 8 (B) consecutive
  // chunks: a single 128-byte wavefront, no bank conflicts.
  constexpr int CW = 16 / sizeof(T);
  constexpr int MCH = TM / CW, NCH = TN / CW;
  constexpr int MSP = 4 * CW, NSP = 8 * CW;  // chunk spacing
  constexpr int VEC = CW;
  static_assert(WARPS_M * WARPS_N == 8, "8 warps");
  static_assert(TM % CW == 0 && TN % CW == 0, "16-byte fragments");

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *As = reinterpret_cast<T *>(smem_raw);
  T *Bs = As + STAGES * BK * BM;

  // Rasterise tiles in groups of 8 along M for L2 reuse of B panels.
  const int tiles_m = (p.m + BM - 1) / BM, tiles_n = (p.n + BN - 1) / BN;
  const int bid = blockIdx.x;
  constexpr int G = 8;
  const int group = bid / (G * tiles_n);
  const int first_m = group * G;
  const int gsize = min(tiles_m - first_m, G);
  const int in_group = bid % (G * tiles_n);
  const int tm = first_m + in_group % gsize, tn = in_group / gsize;
  const long m0 = (long)tm * BM, n0 = (long)tn * BN;

  // block_is_outside(ji, n0, BN, m0, BM)
  if (p.ji == MUBLIS_L3_LOWER && n0 >= m0 + BM) return;
  if (p.ji == MUBLIS_L3_UPPER && n0 + BN <= m0) return;

  long kb = 0, ke = p.k;
  if (p.jp == MUBLIS_L3_LOWER) kb = max(kb, n0);       // j <= p
  if (p.jp == MUBLIS_L3_UPPER) ke = min(ke, n0 + BN);  // j >= p
  if (p.pi == MUBLIS_L3_LOWER) ke = min(ke, m0 + BM);  // p <= i
  if (p.pi == MUBLIS_L3_UPPER) kb = max(kb, m0);       // p >= i
  const int kt_begin = (int)(kb / BK);
  const int kt_end = ke > kb ? (int)((ke + BK - 1) / BK) : kt_begin;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = warp % WARPS_M, wn = warp / WARPS_M;
  const int ty = lane >> 3, tx = lane & 7;

  // PAIR (FP32 only): accumulators as column pairs updated with the packed
  // sm_100 FMA (__ffma2_rn: two correctly rounded fmaf per instruction), so
  // the FMA stream takes half the issue slots and the loads and address
  // arithmetic fit beside it.  Each element's result is that of fmaf.
  static_assert(!PAIR || (sizeof(T) == 4 && TN % 2 == 0), "pairs are FP32 column pairs");
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

  auto load_stage = [&](int stage, int kt) {
    const T *ga = p.ap + (long)kt * BK * p.lda + m0;
    const T *gb = p.bp + (long)kt * BK * p.ldb + n0;
    T *sa = As + stage * BK * BM;
    T *sb = Bs + stage * BK * BN;
#pragma unroll
    for (int c = tid; c < BK * BM / VEC; c += NT) {
      int row = c / (BM / VEC), col = (c % (BM / VEC)) * VEC;
      cp_async16(sa + row * BM + col, ga + (long)row * p.lda + col);
    }
#pragma unroll
    for (int c = tid; c < BK * BN / VEC; c += NT) {
      int row = c / (BN / VEC), col = (c % (BN / VEC)) * VEC;
      cp_async16(sb + row * BN + col, gb + (long)row * p.ldb + col);
    }
  };

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (kt_begin + s < kt_end) load_stage(s, kt_begin + s);
    cp_async_commit();
  }

  for (int kt = kt_begin; kt < kt_end; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int nk = kt + STAGES - 1;
    if (nk < kt_end) load_stage((nk - kt_begin) % STAGES, nk);
    cp_async_commit();

    const int st = (kt - kt_begin) % STAGES;
    const T *sa = As + st * BK * BM + wm * WTM + ty * CW;
    const T *sb = Bs + st * BK * BN + wn * WTN + tx * CW;
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T af[TM], bf[TN];
#pragma unroll
      for (int mc = 0; mc < MCH; ++mc) {
        T t[CW];
        lds16(t, sa + kk * BM + mc * MSP);
#pragma unroll
        for (int q = 0; q < CW; ++q) af[mc * CW + q] = t[q];
      }
#pragma unroll
      for (int nc = 0; nc < NCH; ++nc) {
        T t[CW];
        lds16(t, sb + kk * BN + nc * NSP);
#pragma unroll
        for (int q = 0; q < CW; ++q) bf[nc * CW + q] = t[q];
      }
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TNP; ++j) {
          if constexpr (PAIR)
            acc[i][j] = __ffma2_rn(make_float2(af[i], af[i]), make_float2(bf[2 * j], bf[2 * j + 1]),
                                   acc[i][j]);
          else
            acc[i][j] = fma(af[i], bf[j], acc[i][j]);
        }
    }
  }
  cp_async_wait<0>();

  // Per row, the TN loads of C are issued before the stores (one memory
  // round trip per row rather than per element).
  const T alpha = p.alpha, beta = p.beta;
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const long gi = m0 + wm * WTM + (i / CW) * MSP + ty * CW + (i % CW);
    if (gi >= p.m) continue;
    T cv[TN];
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const long gj = n0 + wn * WTN + (j / CW) * NSP + tx * CW + (j % CW);
      const bool in = gj < p.n && b200_rel(p.ji, gj, gi);
      cv[j] = in && beta != T(0) ? p.c[gi * p.rs_c + gj * p.cs_c] : T(0);
    }
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const long gj = n0 + wn * WTN + (j / CW) * NSP + tx * CW + (j % CW);
      if (gj >= p.n || !b200_rel(p.ji, gj, gi)) continue;
      T v;
      if constexpr (PAIR) v = alpha * ((j & 1) ? acc[i][j >> 1].y : acc[i][j >> 1].x);
      else v = alpha * acc[i][j];
      if (beta != T(0)) v = fma(beta, cv[j], v);
      p.c[gi * p.rs_c + gj * p.cs_c] = v;
    }
  }
}


// Persistent CTAs over (tile, k-chunk) units for split-K calls (SPLIT:
// the split epilogue compiled in).
template <typename T, int BM, int BN, int BK, int WARPS_M, int WARPS_N, int STAGES, int MINB,
          bool PAIR = false, bool SPLIT = false>
__global__ void __launch_bounds__(256, MINB) simt_gemm_kernel(SimtGemmArgs<T> p) {
  constexpr int NT = 256;
  constexpr int WTM = BM / WARPS_M, WTN = BN / WARPS_N;
  constexpr int TM = WTM / 4, TN = WTN / 8;
  // Fragments are 16-byte chunks of CW elements; a thread's chunks are
  // spaced so that one warp-wide load touches 4 (A) or 8 (B) consecutive
  // chunks: a single 128-byte wavefront, no bank conflicts.
  constexpr int CW = 16 / sizeof(T);
  constexpr int MCH = TM / CW, NCH = TN / CW;
  constexpr int MSP = 4 * CW, NSP = 8 * CW;  // chunk spacing
  constexpr int VEC = CW;
  static_assert(WARPS_M * WARPS_N == 8, "8 warps");
  static_assert(TM % CW == 0 && TN % CW == 0, "16-byte fragments");

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *As = reinterpret_cast<T *>(smem_raw);
  T *Bs = As + STAGES * BK * BM;
  __shared__ int s_unit, s_last;

  const int tiles_m = (p.m + BM - 1) / BM, tiles_n = (p.n + BN - 1) / BN;
  const int S = SPLIT ? p.splits : 1;
  const int ntiles = p.ntiles > 0 ? p.ntiles : tiles_m * tiles_n;
  const int units = ntiles * S;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = warp % WARPS_M, wn = warp / WARPS_M;
  const int ty = lane >> 3, tx = lane & 7;

  // PAIR (FP32 only): accumulators as column pairs updated with the packed
  // sm_100 FMA (__ffma2_rn: two correctly rounded fmaf per instruction), so
  // the FMA stream takes half the issue slots and the loads and address
  // arithmetic fit beside it.  Each element's result is that of fmaf.
  static_assert(!PAIR || (sizeof(T) == 4 && TN % 2 == 0), "pairs are FP32 column pairs");
  constexpr int TNP = PAIR ? TN / 2 : TN;
  using Acc = typename std::conditional<PAIR, float2, T>::type;

  // Persistent CTAs take units from p.work; without it, the CTA computes
  // unit blockIdx.x alone.  Unit u is k-chunk u % S of tile u / S.
  int u;
  if (p.work) {
    if (tid == 0) s_unit = atomicAdd(p.work, 1);
    __syncthreads();
    u = s_unit;
  } else {
    u = blockIdx.x;
  }
  while (u < units) {
    const int tslot = u / S, chunk = u % S;
    int tm, tn;
    if (p.tile_list) {
      const int2 t = p.tile_list[tslot];
      tm = t.x;
      tn = t.y;
    } else {
      // Rasterise tiles in groups of 8 along M for L2 reuse of B panels.
      constexpr int G = 8;
      const int group = tslot / (G * tiles_n);
      const int first_m = group * G;
      const int gsize = min(tiles_m - first_m, G);
      const int in_group = tslot % (G * tiles_n);
      tm = first_m + in_group % gsize;
      tn = in_group / gsize;
    }
    const long m0 = (long)tm * BM, n0 = (long)tn * BN;

    // block_is_outside(ji, n0, BN, m0, BM): tile lists hold only tiles that
    // write, so this only skips in the one-tile-per-CTA raster.
    const bool outside = (p.ji == MUBLIS_L3_LOWER && n0 >= m0 + BM) ||
                         (p.ji == MUBLIS_L3_UPPER && n0 + BN <= m0);
    if (!outside) {
      long kb = 0, ke = p.k;
      if (p.jp == MUBLIS_L3_LOWER) kb = max(kb, n0);       // j <= p
      if (p.jp == MUBLIS_L3_UPPER) ke = min(ke, n0 + BN);  // j >= p
      if (p.pi == MUBLIS_L3_LOWER) ke = min(ke, m0 + BM);  // p <= i
      if (p.pi == MUBLIS_L3_UPPER) kb = max(kb, m0);       // p >= i
      const int tile_kt0 = (int)(kb / BK);
      const int tile_kt1 = ke > kb ? (int)((ke + BK - 1) / BK) : tile_kt0;
      // This unit's chunk of the tile's k-blocks (the chunking depends only
      // on the tile's k range and S).
      const int per = (tile_kt1 - tile_kt0 + S - 1) / S;
      const int kt_begin = min(tile_kt1, tile_kt0 + chunk * per);
      const int kt_end = min(tile_kt1, kt_begin + per);

      Acc acc[TM][TNP];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TNP; ++j) {
          if constexpr (PAIR) acc[i][j] = make_float2(0.f, 0.f);
          else acc[i][j] = T(0);
        }

      auto load_stage = [&](int stage, int kt) {
        const T *ga = p.ap + (long)kt * BK * p.lda + m0;
        const T *gb = p.bp + (long)kt * BK * p.ldb + n0;
        T *sa = As + stage * BK * BM;
        T *sb = Bs + stage * BK * BN;
#pragma unroll
        for (int c = tid; c < BK * BM / VEC; c += NT) {
          int row = c / (BM / VEC), col = (c % (BM / VEC)) * VEC;
          cp_async16(sa + row * BM + col, ga + (long)row * p.lda + col);
        }
#pragma unroll
        for (int c = tid; c < BK * BN / VEC; c += NT) {
          int row = c / (BN / VEC), col = (c % (BN / VEC)) * VEC;
          cp_async16(sb + row * BN + col, gb + (long)row * p.ldb + col);
        }
      };

#pragma unroll
      for (int s = 0; s < STAGES - 1; ++s) {
        if (kt_begin + s < kt_end) load_stage(s, kt_begin + s);
        cp_async_commit();
      }

      for (int kt = kt_begin; kt < kt_end; ++kt) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        const int nk = kt + STAGES - 1;
        if (nk < kt_end) load_stage((nk - kt_begin) % STAGES, nk);
        cp_async_commit();

        const int st = (kt - kt_begin) % STAGES;
        const T *sa = As + st * BK * BM + wm * WTM + ty * CW;
        const T *sb = Bs + st * BK * BN + wn * WTN + tx * CW;
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
          T af[TM], bf[TN];
#pragma unroll
          for (int mc = 0; mc < MCH; ++mc) {
            T t[CW];
            lds16(t, sa + kk * BM + mc * MSP);
#pragma unroll
            for (int q = 0; q < CW; ++q) af[mc * CW + q] = t[q];
          }
#pragma unroll
          for (int nc = 0; nc < NCH; ++nc) {
            T t[CW];
            lds16(t, sb + kk * BN + nc * NSP);
#pragma unroll
            for (int q = 0; q < CW; ++q) bf[nc * CW + q] = t[q];
          }
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
      }
      cp_async_wait<0>();

      // Split-K: every chunk stores its sums (element e of thread t at
      // e * 256 + t, so a warp's stores are 128 contiguous bytes); the last
      // chunk of the tile to finish adds all S of them in chunk order --
      // the same order whichever CTA comes last -- and runs the epilogue.
      bool epilogue = true;
      if (SPLIT && S > 1) {
        constexpr int E = TM * TN;
        T *mine = p.partials + (size_t)u * E * NT;
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) {
            T v;
            if constexpr (PAIR) v = (j & 1) ? acc[i][j >> 1].y : acc[i][j >> 1].x;
            else v = acc[i][j];
            mine[(i * TN + j) * NT + tid] = v;
          }
        __threadfence();
        __syncthreads();
        if (tid == 0) s_last = atomicAdd(&p.arrivals[tslot], 1) == S - 1;
        __syncthreads();
        epilogue = s_last;
        if (epilogue) {
          __threadfence();
          const T *first = p.partials + (size_t)tslot * S * E * NT;
#pragma unroll
          for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) {
              T v = __ldcg(first + (i * TN + j) * NT + tid);
              for (int c = 1; c < S; ++c) v += __ldcg(first + ((size_t)c * E + i * TN + j) * NT + tid);
              if constexpr (PAIR) {
                if (j & 1) acc[i][j >> 1].y = v;
                else acc[i][j >> 1].x = v;
              } else {
                acc[i][j] = v;
              }
            }
          if (tid == 0) p.arrivals[tslot] = 0;
        }
      }

      if (epilogue) {
        // Per row, the TN loads of C are issued before the stores (one memory
        // round trip per row rather than per element).
        const T alpha = p.alpha, beta = p.beta;
#pragma unroll
        for (int i = 0; i < TM; ++i) {
          const long gi = m0 + wm * WTM + (i / CW) * MSP + ty * CW + (i % CW);
          if (gi >= p.m) continue;
          T cv[TN];
#pragma unroll
          for (int j = 0; j < TN; ++j) {
            const long gj = n0 + wn * WTN + (j / CW) * NSP + tx * CW + (j % CW);
            const bool in = gj < p.n && b200_rel(p.ji, gj, gi);
            cv[j] = in && beta != T(0) ? p.c[gi * p.rs_c + gj * p.cs_c] : T(0);
          }
#pragma unroll
          for (int j = 0; j < TN; ++j) {
            const long gj = n0 + wn * WTN + (j / CW) * NSP + tx * CW + (j % CW);
            if (gj >= p.n || !b200_rel(p.ji, gj, gi)) continue;
            T v;
            if constexpr (PAIR) v = alpha * ((j & 1) ? acc[i][j >> 1].y : acc[i][j >> 1].x);
            else v = alpha * acc[i][j];
            if (beta != T(0)) v = fma(beta, cv[j], v);
            p.c[gi * p.rs_c + gj * p.cs_c] = v;
          }
        }
      }
    }
    if (!p.work) break;
    __syncthreads();  // shared stages and s_unit are free for the next unit
    if (tid == 0) s_unit = atomicAdd(p.work, 1);
    __syncthreads();
    u = s_unit;
  }
}

template <typename T>
__global__ void scale_kernel(int m, int n, T beta, T *c, long rs, long cs, int ji) {
  long total = (long)m * n;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    long i, j;
    if (rs <= cs) { i = t % m; j = t / m; } else { j = t % n; i = t / n; }
    if (!b200_rel(ji, j, i)) continue;
    T *cij = c + i * rs + j * cs;
    *cij = beta == T(0) ? T(0) : beta * *cij;
  }
}

// Tile configurations: (BM, BN, warps along M, warps along N, cp.async
// stages, min CTAs per SM).  Packed panels are padded to 128 in M and N, so
// every configuration reads the same panels.  Index 0 is the default; the
// others are kept for tuning (MUBLIS_B200_SIMT_S / MUBLIS_B200_SIMT_D).
// Resident CTAs per SM of a kernel at 256 threads and `smem` bytes.
template <typename K>
int resident_per_sm(K kern, size_t smem) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 256, smem) != cudaSuccess || nb < 1)
    nb = 1;
  return nb;
}

template <typename T, int BM, int BN, int WM, int WN, int ST, int MINB, bool PAIR = false>
int launch_cfg(const SimtGemmArgs<T> &a0, cudaStream_t s, const SimtPolicy *pol) {
  constexpr int BK = SimtConfig<T>::BK;
  constexpr int E = (BM / WM / 4) * (BN / WN / 8);  // accumulators per thread
  auto kern = simt_tile_kernel<T, BM, BN, BK, WM, WN, ST, MINB, PAIR>;
  auto kern_split = simt_gemm_kernel<T, BM, BN, BK, WM, WN, ST, MINB, PAIR, true>;
  const size_t smem = (size_t)ST * BK * (BM + BN) * sizeof(T);
  static std::once_flag once;
  static int conf = B200_OK, per_sm = 0;
  B200_TRY(b200_once(once, conf, "gemm: set-up failed", [&]() -> int {
    B200_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    B200_CUDA_TRY(
        cudaFuncSetAttribute(kern_split, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    per_sm = std::min(resident_per_sm(kern, smem), resident_per_sm(kern_split, smem));
    return B200_OK;
  }));
  const long tiles = b200_ceil_div(a0.m, BM) * b200_ceil_div(a0.n, BN);
  if (tiles <= 0) return B200_OK;
  if (tiles > 0x7fffffffL / 16) return b200_set_error(B200_EINVAL, "gemm: too many tiles");
  // Split-K from the whole call's shape (a split unit's 64 KB of partial
  // sums cost about 4 k-block times); unsplit calls take one tile per CTA.
  const long slots = (long)per_sm * b200_sm_count();
  const b200_tile_domain_t dom = {a0.jp, a0.ji, a0.pi};
  const int S = pol ? b200_split_for(pol->m_full, pol->n_full, a0.k, BM, BN, BK, dom, slots, 4.0)
                    : 1;
  if (S == 1) {  // nothing allocated
    B200ProfScope prof(sizeof(T) == 4 ? "simt_sgemm" : "simt_dgemm", s);
    kern<<<(unsigned)tiles, 256, smem, s>>>(a0);
    B200_LAUNCH_CHECK();
    return B200_OK;
  }

  // Persistent CTAs over the tiles that write (heaviest first), each tile's
  // k range cut into S chunks.
  SimtGemmArgs<T> a = a0;
  std::vector<int2> list;
  const bool restricted = a.jp != MUBLIS_L3_ALL || a.ji != MUBLIS_L3_ALL || a.pi != MUBLIS_L3_ALL;
  long ntiles = tiles;
  if (restricted) {
    b200_tile_list(a.m, a.n, a.k, BM, BN, BK, dom, &list, nullptr);
    ntiles = (long)list.size();
    if (ntiles == 0) return B200_OK;
  }
  const long units = ntiles * S;
  const size_t ints = sizeof(int) * (size_t)(1 + ntiles);
  const size_t list_bytes = sizeof(int2) * list.size();
  const size_t part_bytes = S > 1 ? sizeof(T) * (size_t)units * E * 256 : 0;
  char *scratch = nullptr;
  const size_t off_list = b200_round_up((long)ints, 256);
  const size_t off_part = off_list + b200_round_up((long)list_bytes, 256);
  B200_TRY(b200_alloc((void **)&scratch, off_part + part_bytes));
  int st = B200_OK;
  if (cudaMemsetAsync(scratch, 0, ints, s) != cudaSuccess ||
      (list_bytes && cudaMemcpyAsync(scratch + off_list, list.data(), list_bytes,
                                     cudaMemcpyHostToDevice, s) != cudaSuccess))
    st = b200_set_error(B200_ECUDA, "gemm: schedule upload failed");
  if (st == B200_OK) {
    a.work = (int *)scratch;
    a.arrivals = (int *)scratch + 1;
    a.tile_list = restricted ? (const int2 *)(scratch + off_list) : nullptr;
    a.ntiles = (int)ntiles;
    a.splits = S;
    a.partials = S > 1 ? (T *)(scratch + off_part) : nullptr;
    B200ProfScope prof(sizeof(T) == 4 ? "simt_sgemm" : "simt_dgemm", s);
    kern_split<<<(unsigned)std::min(units, slots), 256, smem, s>>>(a);
    if (cudaGetLastError() != cudaSuccess) st = b200_set_error(B200_ECUDA, "gemm: launch failed");
  }
  b200_free(scratch);
  return st;
}

int simt_variant(bool dbl) {
  static int v[2] = {-1, -1};
  if (v[dbl] < 0) {
    const char *e = getenv(dbl ? "MUBLIS_B200_SIMT_D" : "MUBLIS_B200_SIMT_S");
    v[dbl] = e ? atoi(e) : 0;
  }
  return v[dbl];
}

}  // namespace

template <>
int launch_simt_gemm<float>(const SimtGemmArgs<float> &a, cudaStream_t s, const SimtPolicy *pol) {
  switch (simt_variant(false)) {
  case 1: return launch_cfg<float, 128, 128, 2, 4, 4, 2>(a, s, pol);
  case 2: return launch_cfg<float, 128, 128, 4, 2, 3, 1>(a, s, pol);
  case 3: return launch_cfg<float, 128, 128, 4, 2, 4, 2>(a, s, pol);  // scalar fmaf, 4 stages
  case 4: return launch_cfg<float, 128, 128, 4, 2, 4, 2, true>(a, s, pol);  // packed, 4 stages
  // Packed FMA, 2-stage cp.async ring: 52.4 (scalar, 4 stages) -> 58.1 TF/s at 8192^3.
  default: return launch_cfg<float, 128, 128, 4, 2, 2, 2, true>(a, s, pol);
  }
}

template <>
int launch_simt_gemm<double>(const SimtGemmArgs<double> &a, cudaStream_t s, const SimtPolicy *pol) {
  switch (simt_variant(true)) {
  case 1: return launch_cfg<double, 128, 64, 4, 2, 4, 1>(a, s, pol);
  case 2: return launch_cfg<double, 128, 64, 4, 2, 4, 2>(a, s, pol);
  case 3: return launch_cfg<double, 64, 128, 2, 4, 4, 2>(a, s, pol);
  case 4: return launch_cfg<double, 128, 64, 2, 4, 4, 2>(a, s, pol);
  default: return launch_cfg<double, 128, 128, 4, 2, 3, 1>(a, s, pol);  // fastest at n = 4096
  }
}

template <typename T>
int launch_scale(int m, int n, T beta, T *c, long rs, long cs, int ji, cudaStream_t s) {
  if (m <= 0 || n <= 0) return B200_OK;
  long total = (long)m * n;
  unsigned blocks = (unsigned)std::min<long>(b200_ceil_div(total, 256), 148L * 16);
  B200ProfScope prof("scale", s);
  scale_kernel<T><<<blocks, 256, 0, s>>>(m, n, beta, c, rs, cs, ji);
  B200_LAUNCH_CHECK();
  return B200_OK;
}

template int launch_scale<float>(int, int, float, float *, long, long, int, cudaStream_t);
template int launch_scale<double>(int, int, double, double *, long, long, int, cudaStream_t);
