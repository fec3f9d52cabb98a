// gemm_dmma.cu -- plain FP64 GEMM on the FP64 tensor pipe: the device form
// of the reference's five-loop driver (frame/l3/l3_driver.c:126-239) plus
// its micro-kernel (include/mublis_instantiate.h:37-52) for double.
//
// B200 runs FP64 at the same peak on the tensor pipe (mma.sync .f64) as on
// the FMA pipe (37 TF/s).  What the tensor path saves is operand traffic: a
// warp's m16n8k4 MMA takes its 16x4 and 4x8 operands from registers the
// warp loaded once, where an FMA-pipe kernel streams every operand through
// shared memory per thread.  That traffic is what holds the FMA-pipe DGEMM
// well below peak.
//
// Persistent CTAs (one per SM) walk the 128 x 128 output tiles.  Warp 8
// produces: for every k-block of 16 it issues one 16 KB 1-D bulk copy (TMA)
// per operand into a 4-stage shared-memory ring, completing on the stage's
// mbarrier.  The panels are packed in fragment order (PACK_FRAG64), so a
// k-block of a 128-row strip is contiguous and every warp's fragment load
// is 512 contiguous bytes: no swizzle, no bank conflicts.  Warps 0-7
// consume, each a 64 x 32 warp tile (4 x 4 m16n8k4 accumulators, 64 doubles
// a thread), then release the stage to the producer.  Every wait is bounded
// (tc_common.cuh); the producer waits for its own copies before it exits.
//
// Domain handling is the SIMT kernel's: ji skips tiles outside the written
// triangle and masks partial tiles, jp/pi clip each tile's k-range, an empty
// k-range writes beta * C, and beta == 0 never reads C.
#include "kernels.cuh"
#include "tc_common.cuh"

namespace {

constexpr int BM = B200_DMMA_TILE, BN = B200_DMMA_TILE, BK = B200_DMMA_BK, STAGES = 4;
constexpr int CONSUMERS = 8;  // 2 (m) x 4 (n) warps of 64 x 32
constexpr int THREADS = (CONSUMERS + 1) * 32;
constexpr int TILE_BYTES = BM * BK * 8;  // 16 KB per operand per k-block
constexpr int STAGE_BYTES = 2 * TILE_BYTES;
constexpr int SMEM = STAGES * STAGE_BYTES + 128 + 1024;  // + alignment slack for swizzled tiles
constexpr int QUAD_DOUBLES = 8 * 32 * 2;  // one k-quad of a 128-row strip

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

// Tile idx -> (tm, tn): from the host's tile list when the domain
// restricts the output or the k-ranges (only the tiles that write, heaviest
// first, so the strided assignment to persistent CTAs stays balanced), else
// rasterised in groups of 8 along M so that CTAs running together share B
// strips in L2.
__device__ __forceinline__ void tile_coords(const DmmaGemmArgs &p, int idx, int &tm, int &tn) {
  if (p.tile_list) {
    const int2 t = p.tile_list[idx];
    tm = t.x;
    tn = t.y;
    return;
  }
  constexpr int G = 8;
  const int group = idx / (G * p.tiles_n);
  const int first_m = group * G;
  const int gsize = min(p.tiles_m - first_m, G);
  const int in_group = idx % (G * p.tiles_n);
  tm = first_m + in_group % gsize;
  tn = in_group / gsize;
}

// false for a tile wholly outside the written triangle (l3_driver.c:145-147,
// 165-171); else the tile's k-blocks [kt0, kt1) clipped to the product's
// support (:130,148-150,163,171).
__device__ __forceinline__ bool tile_krange(const DmmaGemmArgs &p, int tm, int tn, int &kt0,
                                            int &kt1) {
  const long m0 = (long)tm * BM, n0 = (long)tn * BN;
  if (p.ji == MUBLIS_L3_LOWER && n0 >= m0 + BM) return false;
  if (p.ji == MUBLIS_L3_UPPER && n0 + BN <= m0) return false;
  long kb = 0, ke = p.k;
  if (p.jp == MUBLIS_L3_LOWER) kb = max(kb, n0);       // j <= p
  if (p.jp == MUBLIS_L3_UPPER) ke = min(ke, n0 + BN);  // j >= p
  if (p.pi == MUBLIS_L3_LOWER) ke = min(ke, m0 + BM);  // p <= i
  if (p.pi == MUBLIS_L3_UPPER) kb = max(kb, m0);       // p >= i
  kt0 = (int)(kb / BK);
  kt1 = ke > kb ? (int)((ke + BK - 1) / BK) : kt0;
  return true;
}

// Chunk `chunk` of S of the k-blocks [kt0, kt1) (depends only on the
// tile's k range and S).
__device__ __forceinline__ void chunk_range(int chunk, int S, int &kt0, int &kt1) {
  const int per = (kt1 - kt0 + S - 1) / S;
  const int b = min(kt1, kt0 + chunk * per);
  kt1 = min(kt1, b + per);
  kt0 = b;
}

// Offset (doubles) of element (r, e) of a 128-row x 16 tile stored with the
// 16 innermost: 128-byte rows whose 16-byte chunks are XOR-swizzled by the
// row's low three bits (the TMA 128-byte swizzle).
__device__ __forceinline__ int swz16(int r, int e) {
  return r * 16 + ((((e >> 1) ^ r) & 7) << 1) + (e & 1);
}

// DIRECT: operands come as 2-D TMA tiles of the caller's matrices (A_KC / B_KC:
// k innermost, swizzled [128][16]; else m / n innermost, [16][128]); else
// from PACK_FRAG64 panels by 1-D bulk copies.
template <bool DIRECT, bool A_KC, bool B_KC>
__global__ void __launch_bounds__(THREADS, 1)
    dmma_gemm_kernel(const __grid_constant__ DmmaGemmArgs p) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // Swizzled TMA tiles need 1024-byte aligned destinations.
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(smem + STAGES * STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  volatile int *abort_flag = (volatile int *)(empty + STAGES);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], CONSUMERS);
    }
    *abort_flag = 0;
    tc::fence_barrier_init();
  }
  __syncthreads();
  const int num_tiles = p.tile_list ? p.ntiles : p.tiles_m * p.tiles_n;
  const int S = p.splits;
  const int num_units = num_tiles * S;

  if (warp == CONSUMERS) {
    // ---------------- producer ----------------
    // A stalled launch (armed by mublis_b200_test_stall_next) issues nothing:
    // the consumers' first bounded wait runs out, they raise the abort flag
    // and the error word, and the launch ends with status 4 on the host.
    if (lane != 0 || p.stall) return;
    int stage = 0, issued = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (int u = blockIdx.x; u < num_units && ok; u += gridDim.x) {
      int tm, tn, kt0, kt1;
      tile_coords(p, u / S, tm, tn);
      if (!tile_krange(p, tm, tn, kt0, kt1)) continue;
      chunk_range(u % S, S, kt0, kt1);
      const double *ga = DIRECT ? nullptr : p.ap + (long)tm * p.kq * 2 * 8 * 32;
      const double *gb = DIRECT ? nullptr : p.bp + (long)tn * p.kq * 2 * 8 * 32;
      for (int kt = kt0; kt < kt1; ++kt) {
        if (!tc::mbar_wait(&empty[stage], phase ^ 1, abort_flag, p.err, p.wait_ns)) {
          ok = false;
          break;
        }
        tc::mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
        unsigned char *dst = smem + stage * STAGE_BYTES;
        if constexpr (DIRECT) {
          // The k-block's pair and its k within the pair; the coordinates
          // are multiples of 16 (k) and 128 (m, n), as TMA wants.
          int kl = kt * BK, q = 0;
          if (p.npairs == 2 && kl >= p.kpair) {
            q = 1;
            kl -= (int)p.kpair;
          }
          const int m0 = tm * BM, n0 = tn * BN;
          if (A_KC) tc::tma_load_2d(dst, &p.ta[q], &full[stage], kl, m0);
          else tc::tma_load_2d(dst, &p.ta[q], &full[stage], m0, kl);
          if (B_KC) tc::tma_load_2d(dst + TILE_BYTES, &p.tb[q], &full[stage], kl, n0);
          else tc::tma_load_2d(dst + TILE_BYTES, &p.tb[q], &full[stage], n0, kl);
        } else {
          tc::bulk_load_1d(dst, ga + (long)kt * 4 * QUAD_DOUBLES, TILE_BYTES, &full[stage]);
          tc::bulk_load_1d(dst + TILE_BYTES, gb + (long)kt * 4 * QUAD_DOUBLES, TILE_BYTES,
                           &full[stage]);
        }
        ++issued;
        if (++stage == STAGES) { stage = 0; phase ^= 1; }
      }
    }
    const int pending = issued < STAGES ? issued : STAGES;
    for (int q = 0; q < pending; ++q) {
      if (--stage < 0) { stage = STAGES - 1; phase ^= 1; }
      if (!tc::mbar_wait_drain(&full[stage], phase)) break;
    }
    return;
  }

  // ---------------- consumers ----------------
  const int wm = warp & 1, wn = warp >> 1;
  const int g = lane >> 2, t = lane & 3;
  int stage = 0;
  uint32_t phase = 0;
  for (int u = blockIdx.x; u < num_units; u += gridDim.x) {
    int tm, tn, kt0, kt1;
    tile_coords(p, u / S, tm, tn);
    if (!tile_krange(p, tm, tn, kt0, kt1)) continue;
    chunk_range(u % S, S, kt0, kt1);
    double acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;
    for (int kt = kt0; kt < kt1; ++kt) {
      const int wok = tc::mbar_wait(&full[stage], phase, abort_flag, p.err, p.wait_ns);
      if (!__all_sync(0xffffffffu, wok)) return;
      if constexpr (DIRECT) {
        // Fragments straight from the TMA tiles: a = rows ib*16 + g (+8),
        // k = 4 ks + t of op(A); b = k = 4 ks + t, column jb*8 + g of op(B).
        const double *At = (const double *)(smem + stage * STAGE_BYTES);
        const double *Bt = (const double *)(smem + stage * STAGE_BYTES + TILE_BYTES);
#pragma unroll
        for (int ks = 0; ks < BK / 4; ++ks) {
          const int e = 4 * ks + t;
          double a0[4], a1[4], b[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int r = (wm * 4 + i) * 16 + g;
            a0[i] = A_KC ? At[swz16(r, e)] : At[e * BM + r];
            a1[i] = A_KC ? At[swz16(r + 8, e)] : At[e * BM + r + 8];
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int c = (wn * 4 + j) * 8 + g;
            b[j] = B_KC ? Bt[swz16(c, e)] : Bt[e * BN + c];
          }
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma(acc[i][j], a0[i], a1[i], b[j]);
        }
      } else {
        const double2 *As = (const double2 *)(smem + stage * STAGE_BYTES) + wm * 4 * 32 + lane;
        const double2 *Bs =
            (const double2 *)(smem + stage * STAGE_BYTES + TILE_BYTES) + wn * 2 * 32 + lane;
#pragma unroll
        for (int ks = 0; ks < BK / 4; ++ks) {
          double2 a[4], b[2];
#pragma unroll
          for (int i = 0; i < 4; ++i) a[i] = As[(ks * 8 + i) * 32];
#pragma unroll
          for (int j = 0; j < 2; ++j) b[j] = Bs[(ks * 8 + j) * 32];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
              dmma(acc[i][j], a[i].x, a[i].y, (j & 1) ? b[j >> 1].y : b[j >> 1].x);
        }
      }
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&empty[stage]);
      if (++stage == STAGES) { stage = 0; phase ^= 1; }
    }

    // Split-K: each warp stores its 64 x 32 sums of this chunk (element e of
    // lane l at e * 256 + 32 warp + l: 256 contiguous bytes per warp store);
    // the warp that finishes its sub-tile's last chunk (a per-(tile, warp)
    // counter -- no block-wide barrier, so a warp never waits on another)
    // adds the S chunks' sums in chunk order and runs the epilogue.
    if (S > 1) {
      const int slot = threadIdx.x;  // consumer thread 0..255
      double *mine = p.partials + (size_t)u * 64 * 256;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) mine[((i * 4 + j) * 4 + e) * 256 + slot] = acc[i][j][e];
      __threadfence();
      __syncwarp();
      int last = 0;
      if (lane == 0) last = atomicAdd(&p.arrivals[(u / S) * CONSUMERS + warp], 1) == S - 1;
      last = __shfl_sync(0xffffffffu, last, 0);
      if (!last) continue;
      __threadfence();
      const double *first = p.partials + (size_t)(u / S) * S * 64 * 256;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int off = ((i * 4 + j) * 4 + e) * 256 + slot;
            double v = __ldcg(first + off);
            for (int c = 1; c < S; ++c) v += __ldcg(first + (size_t)c * 64 * 256 + off);
            acc[i][j][e] = v;
          }
      if (lane == 0) p.arrivals[(u / S) * CONSUMERS + warp] = 0;
    }

    // Epilogue: accumulator e of block (i, j) is row g + 8 (e >> 1), column
    // 2 t + (e & 1) of the 16 x 8 block.  The two C values of each pair of
    // adjacent columns are loaded before either is stored: a load / store
    // chain per element pays one memory round trip each (the compiler cannot
    // move a load of C above a store to C).  Larger batches spill at the 168
    // registers a 9-warp CTA allows (measured slower); this one took DGEMM
    // from 32.4 to 33.2 TF/s at 4096^3 and from 34.1 to 34.9 at 8192^3.
    const long m0 = (long)tm * BM + wm * 64, n0 = (long)tn * BN + wn * 32;
    const double alpha = p.alpha, beta = p.beta;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long gi = m0 + i * 16 + g + 8 * h;
        if (gi >= p.m) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          double cv[2];
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const long gj = n0 + j * 8 + 2 * t + e;
            const bool in = gj < p.n && b200_rel(p.ji, gj, gi);
            cv[e] = in && beta != 0.0 ? p.c[gi * p.rs_c + gj * p.cs_c] : 0.0;
          }
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const long gj = n0 + j * 8 + 2 * t + e;
            if (gj >= p.n || !b200_rel(p.ji, gj, gi)) continue;
            double v = alpha * acc[i][j][2 * h + e];
            if (beta != 0.0) v = fma(beta, cv[e], v);
            p.c[gi * p.rs_c + gj * p.cs_c] = v;
          }
        }
      }
  }
}

template <bool DIRECT, bool A_KC, bool B_KC>
int launch_variant(const DmmaGemmArgs &a, int grid, cudaStream_t s) {
  auto kern = dmma_gemm_kernel<DIRECT, A_KC, B_KC>;
  static std::once_flag once;
  static int conf = B200_OK;
  B200_TRY(b200_once(once, conf, "dmma kernel: set-up failed", [&]() -> int {
    B200_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
    return B200_OK;
  }));
  B200ProfScope prof("dmma_dgemm", s);
  kern<<<grid, THREADS, SMEM, s>>>(a);
  B200_LAUNCH_CHECK();
  return B200_OK;
}

}  // namespace

int launch_dmma_gemm(const DmmaGemmArgs &a, cudaStream_t s) {
  const long tiles = (a.tile_list ? a.ntiles : (long)a.tiles_m * a.tiles_n) * a.splits;
  if (tiles <= 0) return B200_OK;
  if (tiles > 0x7fffffffL) return b200_set_error(B200_EINVAL, "dgemm: too many tiles");
  const int sms = b200_sm_count();
  const int grid = (int)(tiles < sms ? tiles : sms);
  if (!a.direct) return launch_variant<false, false, false>(a, grid, s);
  if (a.a_kcontig) {
    return a.b_kcontig ? launch_variant<true, true, true>(a, grid, s)
                       : launch_variant<true, true, false>(a, grid, s);
  }
  return a.b_kcontig ? launch_variant<true, false, true>(a, grid, s)
                     : launch_variant<true, false, false>(a, grid, s);
}
