// tc_grouped.cu -- grouped FP32 GEMMs in the fp16x3 tensor-core form.
//
// The grouped entry points and plans (grouped.cu) use this for 's' problems
// when the FP32 form is fp16x3.  A group is two launches:
//
//  1. tcg_pack_kernel: persistent, one CTA per SM, over strips of 32 rows of
//     op(A) (or 32 columns of op(B)) of one problem with all their k.  A
//     strip lands in shared memory by cp.async two strips ahead of its use
//     (one DRAM read per element); the CTA takes each row's abs-max over k,
//     keeps its scale exponent, and writes the fp16 hi / lo split straight
//     into the byte layout of a 64-byte-swizzled K-major shared-memory tile
//     (the layout a TMA load with 64-byte swizzle produces): 128 rows x 32
//     k, 8 KB per tile and plane.  The main kernel then moves every operand
//     tile with one 1-D bulk copy and needs no tensor map per problem.
//  2. tcg_gemm_kernel: persistent, one CTA per SM, each walking its own list
//     of output tiles (128 rows x BN columns; BN = 16, 32, 64 or 128 by the
//     problem's n), the lists balanced on the host longest-first.  Every
//     tile is one self-contained record (one load per role).  Warp 0 issues
//     the bulk copies into a 6-stage ring, warp 1 issues tcgen05.mma (M =
//     128, N = BN, K = 16) into TMEM, and two epilogue warpgroups take
//     alternate tiles, each with two 128-column TMEM accumulators, so two
//     tiles' write-backs (the latency-bound part of small tiles) overlap
//     each other and the MMAs of the next ones.  Rows past m in a tile's
//     last 8-row group are zero; rows past that are not loaded (their shared
//     memory keeps older data), which only reaches output rows and columns
//     that are never stored.
//
// Numerics are the single-call fp16x3 form's (tc_gemm.cu) step by step: the
// same power-of-two scaling per row of op(A) / column of op(B) over the
// whole k, the same hi / lo split, the same three products in the same order
// per 16-k step, FP32 tensor-core accumulation drained every 256 k into
// round-to-nearest FP32 running sums, and the same epilogue.
#include <cuda_fp16.h>

#include <algorithm>
#include <cstring>
#include <queue>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "tc_common.cuh"
#include "tc_gemm.cuh"

namespace {

constexpr int TCG_BM = 128;                          // rows per output tile
constexpr int TCG_BK = 32;                           // k per k-block (64 bytes of fp16)
constexpr int TCG_ROW = TCG_BK * 2;                  // bytes per tile row
constexpr int TCG_TILE = TCG_BM * TCG_ROW;           // 8 KB: one plane of one tile
constexpr int TCG_STAGES = 6;
constexpr int TCG_STAGE_BYTES = 4 * TCG_TILE;        // A hi, A lo, B hi, B lo
constexpr int TCG_FLUSH = 8;                         // k-blocks per TMEM window (256 k)
constexpr int TCG_ACC_COLS = 128;                    // 2 groups x 2 slots x 128 = 512 columns
constexpr int TCG_THREADS = 384, TCG_GROUP_THREADS = 128;
constexpr int TCG_SMEM = TCG_STAGES * TCG_STAGE_BYTES + 1024 + 256;
constexpr int TCG_PRODUCER_REGS = 56, TCG_EPILOGUE_REGS = 216;
constexpr int TCG_PACK_NBUF = 3;    // strips in the pack ring: two in flight while one is split
constexpr int TCG_PACK_KS = 512;    // k a strip buffer holds; longer rows are read twice
constexpr int TCG_PACK_WARPS = 8;   // warps per pack CTA

// Pack-side view of one problem.
struct TcgProblem {
  int rows_a, rows_b, k, kb;  // m, n, k, ceil(k / 32)
  const float *a;             // op(A)(i, p) at a[i * a_rs + p * a_ks]
  long a_rs, a_ks;
  const float *b;             // op(B)(p, j) at b[j * b_rs + p * b_ks]
  long b_rs, b_ks;
  long a_off, b_off;          // byte offsets of the problem's tiles in the staging areas
  int ea, eb;                 // index of row 0 / column 0 in the exponent array
};

struct TcgPackTask {
  int q, side, row0, pad;  // side 0: rows of op(A); 1: columns of op(B)
};

// Everything one output tile needs.
struct TcgTile {
  long a_src, b_src;     // byte offset of the tile's k-block 0, plane 0, in stage_a / stage_b
  float *c;              // &C(m0, n0)
  long ldc;
  int a_bytes, b_bytes;  // bytes per plane and k-block
  int kb, bn;            // kb = 0: C = beta * C
  int rows, cols;        // valid rows (<= 128) and columns (<= bn)
  float alpha, beta;
  int ea, eb;            // exponent index of the tile's row 0 / column 0
};

__host__ __device__ inline int tcg_rows8(int len, int block) {
  // rows of 128-row block `block` that the staging holds (a multiple of 8)
  const int r = len - block * TCG_BM;
  return r >= TCG_BM ? TCG_BM : (r + 7) & ~7;
}

// Byte offset of (row r, 16-byte chunk ch) in a 64-byte-swizzled tile: the
// chunk index is XORed with address bits 7-8, i.e. (r >> 1) & 3.
__device__ __forceinline__ int tcg_swz(int r, int ch) {
  return r * TCG_ROW + ((ch ^ ((r >> 1) & 3)) << 4);
}

// x * 2^(15 - e) for the fp16 split, as two multiplications by exact
// powers of two: the first is the whole factor whenever 2^(15 - e) is a
// normal float (then it is one rounding of the exact product, as ldexpf
// gives); for rows whose maximum is below 2^-112 the factor is cut in two,
// each scaling up exactly.
__device__ __forceinline__ void tcg_scale_factors(int e, float &f1, float &f2) {
  const int sh = B200_FP16_SCALE_EXP - e;
  const int s1 = sh > 127 ? 127 : (sh < -126 ? -126 : sh);
  f1 = __int_as_float((s1 + 127) << 23);
  f2 = __int_as_float((sh - s1 + 127) << 23);
}

// The scale exponent of b200_scale_exp (frexp's: max|x| < 2^e, 0 for an
// all-zero row) from the bits of a non-negative float, by integer
// arithmetic: normal E - 126, subnormal -117 - clz(mantissa); infinity and
// NaN take b200_scale_exp itself.
__device__ __forceinline__ int tcg_exp_of(unsigned bits) {
  const int E = (int)(bits >> 23);
  if (E == 0) return bits == 0 ? 0 : -117 - __clz((int)bits);
  if (E < 255) return E - 126;
  return b200_scale_exp((unsigned long long)__double_as_longlong((double)__uint_as_float(bits)));
}

// 4-byte asynchronous copy global -> shared (zero-filled when !valid; src
// must still be a valid address).
__device__ __forceinline__ void tcg_cp4(float *dst, const float *src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(tc::smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void tcg_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void tcg_cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

struct TcgStrip {
  const float *x;
  long rs, kst;
  int rows, k, kb, row0, side;
  const TcgProblem *p;
};

__device__ __forceinline__ TcgStrip tcg_strip(const TcgProblem *probs, const TcgPackTask *tasks,
                                              int ti) {
  const TcgPackTask t = tasks[ti];
  const TcgProblem *P = probs + t.q;
  TcgStrip v;
  v.p = P;
  v.side = t.side;
  v.row0 = t.row0;
  v.x = t.side ? P->b : P->a;
  v.rs = t.side ? P->b_rs : P->a_rs;
  v.kst = t.side ? P->b_ks : P->a_ks;
  v.rows = t.side ? P->rows_b : P->rows_a;
  v.k = P->k;
  v.kb = P->kb;
  return v;
}

// buf[r][kk] (row pitch ld) = x(row0 + r, k0 + kk) for kk < w, 0 outside the
// matrix: asynchronous copies (ASYNC) or plain loads.  Lanes run along
// whichever index is contiguous.
template <bool ASYNC>
__device__ __forceinline__ void tcg_fill(const TcgStrip &v, float *buf, int ld, int k0, int w) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int kin = max(0, min(w, v.k - k0));  // strip columns [0, kin) exist in the matrix
  auto put = [&](float *dst, const float *src) {
    if (ASYNC)
      tcg_cp4(dst, src, true);
    else
      *dst = *src;
  };
  if (v.rs == 1 || v.kst != 1) {
    const long gr = (long)v.row0 + lane;
    float *d = buf + lane * ld;
    int kk = warp;
    if (gr < v.rows) {
      const float *src = v.x + gr * v.rs + ((long)k0 + warp) * v.kst;
      const long step = TCG_PACK_WARPS * v.kst;
#pragma unroll 4
      for (; kk < kin; kk += TCG_PACK_WARPS, src += step) put(d + kk, src);
    }
    for (; kk < w; kk += TCG_PACK_WARPS) d[kk] = 0.f;  // past k, or past the matrix's rows
  } else {
    for (int r = warp; r < 32; r += TCG_PACK_WARPS) {
      const long gr = (long)v.row0 + r;
      float *d = buf + r * ld;
      int kk = lane;
      if (gr < v.rows) {
        const float *src = v.x + gr * v.rs + k0 + lane;
#pragma unroll 4
        for (; kk < kin; kk += 32, src += 32) put(d + kk, src);
      }
      for (; kk < w; kk += 32) d[kk] = 0.f;
    }
  }
}

// Persistent: CTA b packs strips b, b + G, b + 2G, ... (G = grid size).  A
// strip is 32 rows of op(A) (or columns of op(B)) of one problem with all of
// their k; strips of up to 512 k go through a ring of three shared-memory
// buffers filled by cp.async two strips ahead; longer ones are read twice
// in 512-k chunks (abs-max, then split).
__global__ void __launch_bounds__(TCG_PACK_WARPS * 32, 1) tcg_pack_kernel(const TcgProblem *__restrict__ probs,
                                                          const TcgPackTask *__restrict__ tasks,
                                                          int ntasks, int ks,
                                                          unsigned char *__restrict__ stage_a,
                                                          unsigned char *__restrict__ stage_b,
                                                          int *__restrict__ exps) {
  extern __shared__ float ring[];  // TCG_PACK_NBUF x 32 x (ks + 1)
  __shared__ unsigned rmax[32];  // bits of each strip row's abs-max (non-negative floats order as ints)
  const int ld = ks + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int mine = ntasks > (int)blockIdx.x ? (ntasks - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto buf_of = [&](int i) { return ring + (i % TCG_PACK_NBUF) * 32 * ld; };
  // Strip descriptors run three ahead in registers, so the dependent loads
  // (task, then problem) of a strip overlap the work on earlier ones.
  auto view = [&](int i) {
    TcgStrip v;
    if (i < mine) return tcg_strip(probs, tasks, (int)blockIdx.x + i * (int)gridDim.x);
    memset(&v, 0, sizeof v);
    return v;
  };
  auto issue = [&](const TcgStrip &v, int i) {  // start strip i's copies (strips that fit a buffer)
    if (i < mine && v.kb * TCG_BK <= ks) tcg_fill<true>(v, buf_of(i), ld, 0, v.kb * TCG_BK);
    tcg_cp_commit();
  };
  if (threadIdx.x < 32) rmax[threadIdx.x] = 0u;
  static_assert(TCG_PACK_NBUF == 3, "the descriptor rotation below assumes a ring of three");
  TcgStrip v0 = view(0), v1 = view(1);
  issue(v0, 0);
  issue(v1, 1);
  TcgStrip v2 = view(2);

  for (int i = 0; i < mine; ++i) {
    issue(v2, i + 2);
    const TcgStrip v3 = view(i + 3);
    const TcgStrip v = v0;
    v0 = v1;
    v1 = v2;
    v2 = v3;
    float *buf = buf_of(i);
    const int kb = v.kb, kpad = kb * TCG_BK;
    const bool resident = kpad <= ks;
    if (resident) {
      tcg_cp_wait<TCG_PACK_NBUF - 1>();  // this strip's group has landed
      __syncthreads();
    }
    // Abs-max of each row over k (lane = row, warp = k residue), folded into
    // rmax by shared-memory atomics (cleared at the end of the previous
    // strip).
    float mx = 0.f;
    for (int k0 = 0; k0 < kpad; k0 += ks) {
      const int w = min(ks, kpad - k0);
      if (!resident) {
        __syncthreads();
        tcg_fill<false>(v, buf, ld, k0, w);
        __syncthreads();
      }
      for (int kk = warp; kk < w; kk += TCG_PACK_WARPS) mx = fmaxf(mx, fabsf(buf[lane * ld + kk]));
    }
    atomicMax(&rmax[lane], __float_as_uint(mx));
    __syncthreads();
    if (threadIdx.x < 32 && v.row0 + lane < v.rows)
      exps[(v.side ? v.p->eb : v.p->ea) + v.row0 + lane] = tcg_exp_of(rmax[lane]);
    // Split and store: item (k-block, row, 16-byte chunk), four consecutive
    // lanes writing one row's 64 bytes.
    const int blk = v.row0 / TCG_BM, r0 = v.row0 % TCG_BM;  // the strip lies in one 128-row block
    const int nr = min(32, tcg_rows8(v.rows, blk) - r0);    // strip rows the staging holds
    unsigned char *tiles0 = (v.side ? stage_b + v.p->b_off : stage_a + v.p->a_off) +
                            (long)blk * kb * 2 * TCG_TILE;
    for (int k0 = 0; k0 < kpad; k0 += ks) {
      const int w = min(ks, kpad - k0);
      if (!resident) {
        __syncthreads();
        tcg_fill<false>(v, buf, ld, k0, w);
        __syncthreads();
      }
      const int items = (w / TCG_BK) * 128;
      for (int it = threadIdx.x; it < items; it += TCG_PACK_WARPS * 32) {
        const int ch = it & 3, r = (it >> 2) & 31, cl = it >> 7;
        if (r >= nr) continue;
        float f1, f2;
        tcg_scale_factors(tcg_exp_of(rmax[r]), f1, f2);
        const float *src = buf + r * ld + cl * TCG_BK + ch * 8;
        __align__(16) __half2 h[4], l[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {  // two elements per conversion
          const float a = (src[2 * j] * f1) * f2, b = (src[2 * j + 1] * f1) * f2;
          h[j] = __floats2half2_rn(a, b);
          const float2 hf = __half22float2(h[j]);
          l[j] = __floats2half2_rn(a - hf.x, b - hf.y);
        }
        unsigned char *dst =
            tiles0 + ((long)(k0 / TCG_BK + cl) * 2) * TCG_TILE + tcg_swz(r0 + r, ch);
        *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<const uint4 *>(h);
        *reinterpret_cast<uint4 *>(dst + TCG_TILE) = *reinterpret_cast<const uint4 *>(l);
      }
    }
    __syncthreads();  // the buffer is free for the strip issued next iteration
    if (threadIdx.x < 32) rmax[threadIdx.x] = 0u;  // read by no one until the next barrier
  }
  tcg_cp_wait<0>();
}

__global__ void __launch_bounds__(TCG_THREADS, 1)
    tcg_gemm_kernel(const TcgTile *__restrict__ tiles, const int *__restrict__ cta_start,
                    const unsigned char *__restrict__ stage_a,
                    const unsigned char *__restrict__ stage_b, const int *__restrict__ exps,
                    int *err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem = (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(smem + TCG_STAGES * TCG_STAGE_BYTES);
  uint64_t *empty = full + TCG_STAGES;
  uint64_t *tfull = empty + TCG_STAGES;  // per accumulator slot (group g: slots 2g, 2g+1)
  uint64_t *tempty = tfull + 4;
  uint64_t *drain = tempty + 4;
  uint32_t *tmem_slot = (uint32_t *)(drain + 1);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < TCG_STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 4; ++a) {
      tc::mbar_init(&tfull[a], 1);
      tc::mbar_init(&tempty[a], TCG_GROUP_THREADS);
    }
    tc::mbar_init(drain, 1);
    *abort_flag = 0;
    tc::fence_barrier_init();
  }
  if (warp == 2) tc::tmem_alloc(tmem_slot, 4 * TCG_ACC_COLS);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const int t0 = cta_start[blockIdx.x], t1 = cta_start[blockIdx.x + 1];
  auto sa = [&](int s, int t) { return smem + s * TCG_STAGE_BYTES + t * TCG_TILE; };
  auto sb = [&](int s, int t) { return smem + s * TCG_STAGE_BYTES + (2 + t) * TCG_TILE; };

  // Register split (as in the single-call kernels): warpgroup 0 drops, the
  // epilogue warpgroups rise for the 128 running sums per thread.
  if (warp < 4) {
  tc::setmaxnreg_dec<TCG_PRODUCER_REGS>();
  if (warp == 0 && lane == 0) {
    // ---------------- bulk-copy producer ----------------
    int stage = 0, issued = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (int ti = t0; ti < t1 && ok; ++ti) {
      const int kb = tiles[ti].kb;
      if (kb == 0) continue;
      const unsigned char *ab = stage_a + tiles[ti].a_src;
      const unsigned char *bb = stage_b + tiles[ti].b_src;
      const uint32_t a_bytes = tiles[ti].a_bytes, b_bytes = tiles[ti].b_bytes;
      for (int c = 0; c < kb; ++c) {
        if (!tc::mbar_wait(&empty[stage], phase ^ 1, abort_flag, err)) { ok = false; break; }
        tc::mbar_arrive_expect_tx(&full[stage], 2 * (a_bytes + b_bytes));
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          tc::bulk_load_1d(sa(stage, t), ab + ((long)c * 2 + t) * TCG_TILE, a_bytes, &full[stage]);
          tc::bulk_load_1d(sb(stage, t), bb + ((long)c * 2 + t) * TCG_TILE, b_bytes, &full[stage]);
        }
        ++issued;
        if (++stage == TCG_STAGES) { stage = 0; phase ^= 1; }
      }
    }
    // Drain: wait (bounded) for the copies of the last ring's worth of stages.
    int pending = issued < TCG_STAGES ? issued : TCG_STAGES;
    for (int q = 0; q < pending; ++q) {
      if (--stage < 0) { stage = TCG_STAGES - 1; phase ^= 1; }
      if (!tc::mbar_wait_drain(&full[stage], phase)) break;
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    int stage = 0;
    uint32_t phase = 0;
    // Accumulator slot state per epilogue group g, packed as bits: bit g =
    // slot within the group's pair, bit 2 + g = that pair's phase.
    uint32_t sst = 0;
    bool ok = true, any = false;
    for (int ti = t0; ti < t1 && ok; ++ti) {
      const int g = (ti - t0) & 1;
      const int kb = tiles[ti].kb;
      const uint32_t idesc = tc::idesc_f16(TCG_BM, tiles[ti].bn);
      for (int c0 = 0; c0 < kb && ok; c0 += TCG_FLUSH) {
        const int c1 = min(kb, c0 + TCG_FLUSH);
        const int s = 2 * g + (int)((sst >> g) & 1);
        const uint32_t sph = (sst >> (2 + g)) & 1;
        if (!tc::mbar_wait(&tempty[s], sph ^ 1, abort_flag, err)) { ok = false; break; }
        tc::tc_fence_after();
        const uint32_t d = tmem_base + (uint32_t)(s * TCG_ACC_COLS);
        for (int c = c0; c < c1; ++c) {
          if (!tc::mbar_wait(&full[stage], phase, abort_flag, err)) { ok = false; break; }
          tc::tc_fence_after();
          const uint64_t ah = tc::smem_desc(sa(stage, 0), 64), al = tc::smem_desc(sa(stage, 1), 64);
          const uint64_t bh = tc::smem_desc(sb(stage, 0), 64), bl = tc::smem_desc(sb(stage, 1), 64);
#pragma unroll
          for (int ks = 0; ks < 2; ++ks) {
            const uint64_t o = (uint64_t)((ks * 32) >> 4);
            // small terms first, the hi * hi product last
            tc::mma_bf16(d, ah + o, bl + o, idesc, c == c0 && ks == 0 ? 0u : 1u);
            tc::mma_bf16(d, al + o, bh + o, idesc, 1u);
            tc::mma_bf16(d, ah + o, bh + o, idesc, 1u);
          }
          tc::mma_commit(&empty[stage]);
          any = true;
          if (++stage == TCG_STAGES) { stage = 0; phase ^= 1; }
        }
        if (!ok) break;
        tc::mma_commit(&tfull[s]);
        sst ^= 1u << g;                              // next slot of the pair
        if (((sst >> g) & 1) == 0) sst ^= 4u << g;   // wrapped: next phase
      }
    }
    if (any) {  // every issued MMA has completed before TMEM is released
      tc::mma_commit(drain);
      tc::mbar_wait(drain, 0, abort_flag, err);
    }
  }
  } else {
    tc::setmaxnreg_inc<TCG_EPILOGUE_REGS>();
    // ---------------- epilogue: group g takes tiles t0 + g, t0 + g + 2, ... ----------------
    const int g = (warp - 4) >> 2;
    const int quad = warp & 3;  // TMEM lanes 32*quad .. 32*quad+31
    const int row = quad * 32 + lane;
    const uint32_t lane_base = tmem_base + ((uint32_t)(quad * 32) << 16);
    int slot = 0;
    uint32_t sphase = 0;
    bool ok = true;
    float run[128];
    for (int ti = t0 + g; ti < t1 && ok; ti += 2) {
      const TcgTile &T = tiles[ti];
      const int kb = T.kb, bn = T.bn, cols = T.cols;
      const bool row_ok = row < T.rows;
      const long ldc = T.ldc;
      const float alpha = T.alpha, beta = T.beta;
      float *crow = T.c + row;
      if (kb == 0) {  // no update: beta * C
        if (row_ok)
          for (int j = 0; j < cols; ++j) {
            float *cij = crow + j * ldc;
            *cij = beta != 0.f ? beta * *cij : 0.f;
          }
        continue;
      }
      if (row_ok && beta != 0.f)  // pull this row's C into L2 while the MMAs run
        for (int j = 0; j < cols; ++j)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(crow + j * ldc));
      const int nwin = (kb + TCG_FLUSH - 1) / TCG_FLUSH;
      const int *ej = exps + T.eb;
      if (nwin == 1) {
        // One window: drain and write back 16 columns at a time straight
        // from TMEM, holding the slot until the tile is written (the
        // group's other slot takes the MMAs of its next tile meanwhile).
        const int s = 2 * g + slot;
        int wok = tc::mbar_wait(&tfull[s], sphase, abort_flag, err);
        if (!__all_sync(0xffffffffu, wok)) { ok = false; break; }
        tc::tc_fence_after();
        const uint32_t base = lane_base + (uint32_t)(s * TCG_ACC_COLS);
        const int ei = row_ok ? exps[T.ea + row] : 0;
        int echunk = 0;
#pragma unroll 1
        for (int j0 = 0; j0 < cols; j0 += 16) {
          if ((j0 & 31) == 0) echunk = j0 + lane < cols ? ej[j0 + lane] : 0;
          float cv[16];
#pragma unroll
          for (int j = 0; j < 16; ++j)
            cv[j] = row_ok && j0 + j < cols && beta != 0.f ? crow[(j0 + j) * ldc] : 0.f;
          uint32_t r[16];
          tc::tmem_ld16(base + (uint32_t)j0, r);
          tc::tmem_wait_ld();
          tc::tmem_tie16(r);
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int fj = __shfl_sync(0xffffffffu, echunk, (j0 & 31) + j);
            if (!row_ok || j0 + j >= cols) continue;
            float v = alpha * b200_pow2_scale(__uint_as_float(r[j]),
                                              ei + fj - 2 * B200_FP16_SCALE_EXP);
            if (beta != 0.f) v = fmaf(beta, cv[j], v);
            crow[(j0 + j) * ldc] = v;
          }
        }
        tc::tc_fence_before();
        tc::mbar_arrive(&tempty[s]);
        if ((slot ^= 1) == 0) sphase ^= 1;
        continue;
      }
      for (int win = 0; win < nwin; ++win) {
        const int s = 2 * g + slot;
        // Every lane observes the barrier; the outcome is made warp-uniform
        // because the TMEM loads below are .sync.aligned.
        int wok = tc::mbar_wait(&tfull[s], sphase, abort_flag, err);
        if (!__all_sync(0xffffffffu, wok)) { ok = false; break; }
        tc::tc_fence_after();
        const uint32_t base = lane_base + (uint32_t)(s * TCG_ACC_COLS);
        // One 16-column TMEM load at a time (the 128 running sums leave no
        // registers for more in flight).
#pragma unroll
        for (int g0 = 0; g0 < 8; ++g0) {
          if (g0 * 16 >= bn) break;
          uint32_t r[16];
          tc::tmem_ld16(base + (uint32_t)(g0 * 16), r);
          tc::tmem_wait_ld();
          tc::tmem_tie16(r);
#pragma unroll
          for (int j = 0; j < 16; ++j)
            run[g0 * 16 + j] = win == 0 ? __uint_as_float(r[j])
                                        : __fadd_rn(run[g0 * 16 + j], __uint_as_float(r[j]));
        }
        tc::tc_fence_before();
        tc::mbar_arrive(&tempty[s]);
        if ((slot ^= 1) == 0) sphase ^= 1;
      }
      if (!ok) break;
      // Write-back in 16-column batches: the batch's C loads are issued
      // before its stores.  Lane j of each warp holds the exponent of
      // column j0 + j of a 32-column chunk, broadcast by shuffles (all lanes
      // take part; rows past the tile only skip their loads and stores).
      const int ei = row_ok ? exps[T.ea + row] : 0;
      int echunk = 0;
#pragma unroll
      for (int j0 = 0; j0 < 128; j0 += 16) {
        if (j0 >= cols) break;
        if ((j0 & 31) == 0) echunk = j0 + lane < cols ? ej[j0 + lane] : 0;
        float cv[16];
#pragma unroll
        for (int j = 0; j < 16; ++j)
          cv[j] = row_ok && j0 + j < cols && beta != 0.f ? crow[(j0 + j) * ldc] : 0.f;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int fj = __shfl_sync(0xffffffffu, echunk, (j0 & 31) + j);
          if (!row_ok || j0 + j >= cols) continue;
          float v = alpha * b200_pow2_scale(run[j0 + j], ei + fj - 2 * B200_FP16_SCALE_EXP);
          if (beta != 0.f) v = fmaf(beta, cv[j], v);
          crow[(j0 + j) * ldc] = v;
        }
      }
    }
  }

  tc::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem_base, 4 * TCG_ACC_COLS);
  }
}

int tcg_bn(int n) { return n <= 16 ? 16 : n <= 32 ? 32 : n <= 64 ? 64 : 128; }

}  // namespace

struct b200_tcg {
  void *mem = nullptr;
  TcgProblem *probs = nullptr;
  TcgTile *tiles = nullptr;
  int *cta_start = nullptr;
  TcgPackTask *tasks = nullptr;
  int *exps = nullptr;
  unsigned char *stage_a = nullptr, *stage_b = nullptr;
  int ntasks = 0, ntiles = 0, grid = 0, kpad_max = TCG_BK;
};

int b200_tcg_create(const mublis_b200_gemm_problem_t *p, int count, b200_tcg **out) {
  *out = nullptr;
  std::vector<TcgProblem> probs;
  std::vector<TcgTile> tiles;
  std::vector<long> cost;
  std::vector<TcgPackTask> tasks;
  long a_bytes = 0, b_bytes = 0, nexp = 0;
  int kpad_max = TCG_BK;
  for (int q = 0; q < count; ++q) {
    const mublis_b200_gemm_problem_t &x = p[q];
    if (x.m < 0 || x.n < 0 || x.k < 0) return b200_set_error(B200_EINVAL, "grouped gemm: negative size");
    if (x.m == 0 || x.n == 0) continue;
    if (x.ldc < std::max(1, x.m)) return b200_set_error(B200_EINVAL, "grouped gemm: ldc too small");
    const bool upd = x.alpha != 0.0 && x.k > 0;
    if (!b200_is_device_ptr(x.c) || (upd && (!b200_is_device_ptr(x.a) || !b200_is_device_ptr(x.b))))
      return b200_set_error(B200_EINVAL, "grouped gemm: operands must be device pointers");
    const int k = upd ? x.k : 0, kb = (int)b200_ceil_div(k, TCG_BK);
    const int mt = (int)b200_ceil_div(x.m, TCG_BM), nt128 = (int)b200_ceil_div(x.n, TCG_BM);
    TcgProblem e;
    memset(&e, 0, sizeof e);
    if (kb > 0) {
      if (nexp + (long)x.m + x.n > 0x7fffffffL)
        return b200_set_error(B200_EINVAL, "grouped gemm: too many rows in the group");
      e.rows_a = x.m;
      e.rows_b = x.n;
      e.k = k;
      e.kb = kb;
      e.a = (const float *)x.a;
      e.a_rs = x.trans_a == MUBLIS_TRANSPOSE ? x.lda : 1;
      e.a_ks = x.trans_a == MUBLIS_TRANSPOSE ? 1 : x.lda;
      e.b = (const float *)x.b;
      e.b_rs = x.trans_b == MUBLIS_TRANSPOSE ? 1 : x.ldb;
      e.b_ks = x.trans_b == MUBLIS_TRANSPOSE ? x.ldb : 1;
      e.a_off = a_bytes;
      e.b_off = b_bytes;
      e.ea = (int)nexp;
      e.eb = (int)(nexp + x.m);
      a_bytes += (long)mt * kb * 2 * TCG_TILE;
      b_bytes += (long)nt128 * kb * 2 * TCG_TILE;
      nexp += (long)x.m + x.n;
      kpad_max = std::max(kpad_max, kb * TCG_BK);
      for (int r = 0; r < x.m; r += 32) tasks.push_back(TcgPackTask{(int)probs.size(), 0, r, 0});
      for (int r = 0; r < x.n; r += 32) tasks.push_back(TcgPackTask{(int)probs.size(), 1, r, 0});
      probs.push_back(e);
    }
    const int bn = tcg_bn(x.n);
    for (int tm = 0; tm < mt; ++tm)
      for (int n0 = 0; n0 < x.n; n0 += bn) {
        TcgTile t;
        memset(&t, 0, sizeof t);
        const int m0 = tm * TCG_BM, bblk = n0 / TCG_BM, sub = n0 % TCG_BM;
        t.kb = kb;
        t.bn = bn;
        t.rows = std::min(TCG_BM, x.m - m0);
        t.cols = std::min(bn, x.n - n0);
        t.c = (float *)x.c + m0 + (long)n0 * x.ldc;
        t.ldc = x.ldc;
        t.alpha = (float)x.alpha;
        t.beta = (float)x.beta;
        if (kb > 0) {
          t.a_src = e.a_off + (long)tm * kb * 2 * TCG_TILE;
          t.b_src = e.b_off + (long)bblk * kb * 2 * TCG_TILE + (long)sub * TCG_ROW;
          t.a_bytes = tcg_rows8(x.m, tm) * TCG_ROW;
          t.b_bytes = std::min(bn, tcg_rows8(x.n, bblk) - sub) * TCG_ROW;
          t.ea = e.ea + m0;
          t.eb = e.eb + n0;
        }
        tiles.push_back(t);
        // copy-bound estimate: rows moved per k-block, plus the write-back
        cost.push_back((long)kb * (tcg_rows8(x.m, tm) + bn) + 4L * bn + 64);
      }
  }
  if (tiles.size() > 0x7fffffffL || tasks.size() > 0x7fffffffL)
    return b200_set_error(B200_EINVAL, "grouped gemm: too many tiles");
  auto *g = new b200_tcg;
  g->ntiles = (int)tiles.size();
  g->ntasks = (int)tasks.size();
  g->grid = std::min(g->ntiles, b200_sm_count());
  g->kpad_max = kpad_max;
  // Longest tile first onto the least-loaded CTA; each CTA's list keeps
  // that order.
  std::vector<int> order(tiles.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  std::vector<std::vector<int>> lists(g->grid);
  using Load = std::pair<long, int>;
  std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
  for (int b = 0; b < g->grid; ++b) heap.push(Load{0, b});
  for (int i : order) {
    Load l = heap.top();
    heap.pop();
    lists[l.second].push_back(i);
    heap.push(Load{l.first + cost[i], l.second});
  }
  std::vector<TcgTile> flat;
  std::vector<int> start(g->grid + 1, 0);
  flat.reserve(tiles.size());
  for (int b = 0; b < g->grid; ++b) {
    start[b] = (int)flat.size();
    for (int i : lists[b]) flat.push_back(tiles[i]);
  }
  start[g->grid] = (int)flat.size();
  // One device allocation: tables, exponents and both staging areas.
  auto al = [](long x) { return b200_round_up(x, 256); };
  const long o_probs = 0, o_tiles = o_probs + al(sizeof(TcgProblem) * probs.size());
  const long o_start = o_tiles + al(sizeof(TcgTile) * flat.size());
  const long o_tasks = o_start + al(sizeof(int) * start.size());
  const long o_exps = o_tasks + al(sizeof(TcgPackTask) * tasks.size());
  const long o_a = o_exps + al(sizeof(int) * nexp);
  const long o_b = o_a + al(a_bytes);
  const long total = o_b + al(b_bytes);
  const long table_bytes = o_exps;
  cudaStream_t s = b200_cur_stream();
  int st = b200_alloc(&g->mem, (size_t)std::max(total, 256L));
  if (st == B200_OK) {
    unsigned char *base = (unsigned char *)g->mem;
    g->probs = (TcgProblem *)(base + o_probs);
    g->tiles = (TcgTile *)(base + o_tiles);
    g->cta_start = (int *)(base + o_start);
    g->tasks = (TcgPackTask *)(base + o_tasks);
    g->exps = (int *)(base + o_exps);
    g->stage_a = base + o_a;
    g->stage_b = base + o_b;
    std::vector<unsigned char> host((size_t)table_bytes, 0);
    if (!probs.empty()) memcpy(host.data() + o_probs, probs.data(), sizeof(TcgProblem) * probs.size());
    if (!flat.empty()) memcpy(host.data() + o_tiles, flat.data(), sizeof(TcgTile) * flat.size());
    memcpy(host.data() + o_start, start.data(), sizeof(int) * start.size());
    if (!tasks.empty()) memcpy(host.data() + o_tasks, tasks.data(), sizeof(TcgPackTask) * tasks.size());
    if (table_bytes > 0 &&
        cudaMemcpyAsync(g->mem, host.data(), (size_t)table_bytes, cudaMemcpyHostToDevice, s) !=
            cudaSuccess)
      st = b200_set_error(B200_ECUDA, "grouped gemm: table upload failed");
    // The host image must outlive the copy.
    if (st == B200_OK && cudaStreamSynchronize(s) != cudaSuccess)
      st = b200_set_error(B200_ECUDA, "grouped gemm: table upload failed");
  }
  if (st != B200_OK) {
    b200_tcg_destroy(g);
    return st;
  }
  *out = g;
  return B200_OK;
}

int b200_tcg_run(b200_tcg *g, cudaStream_t s) {
  static std::once_flag once;
  static int conf = B200_OK;
  B200_TRY(b200_once(once, conf, "grouped fp16x3 kernels: set-up failed", []() -> int {
    B200_CUDA_TRY(cudaFuncSetAttribute(tcg_pack_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(sizeof(float) * TCG_PACK_NBUF * 32 * (TCG_PACK_KS + 1))));
    B200_CUDA_TRY(cudaFuncSetAttribute(tcg_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       TCG_SMEM));
    // The register split needs 128 x (R - 56) >= 256 x (216 - R) at the
    // compiled allocation R; an increase that cannot be granted waits
    // forever, so refuse to launch instead.
    cudaFuncAttributes fa;
    B200_CUDA_TRY(cudaFuncGetAttributes(&fa, tcg_gemm_kernel));
    if (fa.numRegs < TCG_PRODUCER_REGS ||
        128L * (fa.numRegs - TCG_PRODUCER_REGS) < 256L * (TCG_EPILOGUE_REGS - fa.numRegs))
      return b200_set_error(B200_EINVAL, "grouped fp16x3 kernel: register split does not fit");
    return B200_OK;
  }));
  if (g->ntasks > 0) {
    const int ks = std::min(g->kpad_max, TCG_PACK_KS);
    const size_t smem = sizeof(float) * TCG_PACK_NBUF * 32 * (ks + 1);
    const int grid = std::min(g->ntasks, b200_sm_count());
    B200ProfScope prof("tcg_pack", s);
    tcg_pack_kernel<<<grid, TCG_PACK_WARPS * 32, smem, s>>>(g->probs, g->tasks, g->ntasks, ks, g->stage_a,
                                            g->stage_b, g->exps);
    B200_LAUNCH_CHECK();
  }
  if (g->ntiles > 0) {
    B200ProfScope prof("tcg_fp16x3", s);
    tcg_gemm_kernel<<<g->grid, TCG_THREADS, TCG_SMEM, s>>>(g->tiles, g->cta_start, g->stage_a,
                                                           g->stage_b, g->exps,
                                                           b200_device_error_word());
    B200_LAUNCH_CHECK();
  }
  return B200_OK;
}

void b200_tcg_destroy(b200_tcg *g) {
  if (!g) return;
  b200_free(g->mem);
  delete g;
}
