// trsm_leaf.cu -- the fused GEMMTRSM kernel: solves one leaf of a left
// triangular solve (up to 512 rows, every right-hand side) in one launch,
// the diagonal blocks by substitution in shared memory and the updates
// between them on the FP64 tensor pipe.
//
// Reference: the blocked solve of frame/l3/trsm.c:139-183 calls the
// gemmtrsm{l,u} micro-kernel (include/mublis_instantiate.h:95-114,
// targets/avx2/gemmtrsm_ukr.inc:95-215), which forms B11 - A1x * Bx1 and
// solves the MR x MR diagonal block A11 (packed with its diagonal already
// inverted, packm.c:143-144) in registers.  Here one CTA owns 32
// right-hand-side columns of a leaf of 512 rows and keeps the whole 512 x 32
// block of B in registers (8 warps, each 4 row blocks of 16 rows, assigned
// cyclically so that every warp keeps working as the solve moves down).  For
// each diagonal block d of 16 rows:
//   * the warp that owns block d + 1 first applies block d's update to it,
//     then solves it in shared memory, X = inv(D) R with the inverse of its
//     16 x 16 diagonal block -- so the next block is ready by the time the
//     other warps finish their updates (look-ahead);
//   * every other warp applies X_d to its blocks below: B_rb -= A_rb,d X_d,
//     16 x 32 x 16 per block as m16n8k4 .f64 MMAs on the tensor pipe;
//   * all threads write X_d to B (off the owner's critical path).
// One barrier per block.  The leaf's A is packed once per solve
// (trsm_leaf_pack_kernel) into one contiguous segment per step -- the
// column of 16 x 16 blocks below the diagonal block in MMA fragment order,
// then the inverse of the next diagonal block, formed by substitution
// against the reciprocal diagonal (the reference's inverted-diagonal
// packing, packm.c:143-144, carried to the whole 16 x 16 block) -- and one
// thread streams segments into a 3-deep shared-memory ring with 1-D bulk
// copies (TMA), two steps ahead.  Every wait is bounded (tc_common.cuh); a
// CTA that gives up waits for its own copies and returns, and the call
// reports status 4.
//
// An upper-triangular leaf is the lower one with rows and columns reversed:
// the pack reads A from the bottom-right corner and the kernel addresses B
// from the leaf's last row with a negated row stride.
#include <type_traits>

#include "kernels.cuh"
#include "tc_common.cuh"

namespace {

constexpr int LB = 16;                     // rows of a diagonal block
constexpr int LEAF_BLOCKS = 32;            // diagonal blocks per leaf
constexpr int BLK = LB * LB;               // elements of a packed 16 x 16 block
constexpr int NBC = 32;                    // right-hand-side columns per CTA
constexpr int XS_LD = 40;                  // padded row of a solved block in smem
constexpr int SEG_MAX = LEAF_BLOCKS * BLK; // largest segment: 31 panel blocks + 1 diagonal block
constexpr int RING = 3;
constexpr int THREADS = 256;

// Offset (elements) of step d's segment in a leaf of nb blocks: the leaf
// starts with diagonal block 0, then segment d = (nb - 1 - d) panel blocks
// and diagonal block d + 1, for d = 0 .. nb - 2.
__host__ __device__ inline long seg_off(int d, int nb) {
  return (long)BLK * (1 + (long)d * nb - (long)d * (d - 1) / 2);
}

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double b0) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(b0));
}

struct LeafPackArgs {
  const void *a;
  long rs_a, cs_a;
  int m;          // order of the whole solve
  int leaf_rows;  // 512
  int lower, unit;
  void *out;
  long leaf_stride;  // elements per packed leaf
};

// Element (i, p) of a leaf in lower orientation (rows r0 .. r0 + rows); the
// identity outside it; the stored diagonal replaced by its reciprocal (or 1
// for a unit diagonal); the unstored triangle never read.
template <typename T>
__device__ T leaf_elem(const LeafPackArgs &a, long r0, int rows, int i, int p) {
  if (i >= rows || p >= rows) return i == p ? T(1) : T(0);
  if (p > i) return T(0);
  const long ri = a.lower ? r0 + i : r0 + rows - 1 - i;
  const long pj = a.lower ? r0 + p : r0 + rows - 1 - p;
  const T *x = (const T *)a.a;
  if (i == p) return a.unit ? T(1) : T(1) / x[ri * a.rs_a + pj * a.cs_a];
  return x[ri * a.rs_a + pj * a.cs_a];
}

// grid (LEAF_BLOCKS, leaves * LEAF_BLOCKS), 256 threads: blockIdx.y =
// leaf * LEAF_BLOCKS + s; s = 0 is diagonal block 0, s = d + 1 is step d's
// segment, whose block x is panel block d + 1 + x or, for the last x, the
// inverse of diagonal block d + 1.  FP64 blocks are stored in MMA
// A-fragment order; FP32 panel blocks column-major, inverses row-major.
template <typename T>
__global__ void __launch_bounds__(256) trsm_leaf_pack_kernel(const LeafPackArgs a) {
  __shared__ T tile[LB][LB + 1];
  const int leaf = blockIdx.y / LEAF_BLOCKS, s = blockIdx.y % LEAF_BLOCKS, x = blockIdx.x;
  const long r0 = (long)leaf * a.leaf_rows;
  const int rows = (int)min((long)a.leaf_rows, a.m - r0);
  const int nb = (rows + LB - 1) / LB;
  int bi, bp;  // block coordinates in the leaf
  bool diag;
  long off;
  if (s == 0) {
    if (x > 0) return;
    bi = bp = 0;
    diag = true;
    off = 0;
  } else {
    const int d = s - 1;
    if (d > nb - 2 || x > nb - 1 - d) return;
    diag = x == nb - 1 - d;
    bi = diag ? d + 1 : d + 1 + x;
    bp = diag ? d + 1 : d;
    off = seg_off(d, nb) + (long)x * BLK;
  }
  const int tid = threadIdx.x;
  // Read with the stored matrix's unit stride running across the warp.
  const bool rows_fast = labs(a.rs_a) <= labs(a.cs_a);
  const int ri = rows_fast ? tid % LB : tid / LB, pi = rows_fast ? tid / LB : tid % LB;
  tile[ri][pi] = leaf_elem<T>(a, r0, rows, bi * LB + ri, bp * LB + pi);
  __syncthreads();
  if (diag) {
    // The block's inverse, column j by thread j: forward substitution
    // L x = e_j against the reciprocal diagonal (tile[i][i] = 1 / a_ii, as
    // the reference packs it, packm.c:143-144).
    T x[LB];
    if (tid < LB) {
#pragma unroll
      for (int i = 0; i < LB; ++i) {
        T r = i == tid ? T(1) : T(0);
#pragma unroll
        for (int q = 0; q < i; ++q) r = fma(-tile[i][q], x[q], r);
        x[i] = r * tile[i][i];
      }
    }
    __syncthreads();
    if (tid < LB) {
#pragma unroll
      for (int i = 0; i < LB; ++i) tile[i][tid] = x[i];
    }
    __syncthreads();
  }
  T *out = (T *)a.out + (long)leaf * a.leaf_stride + off;
  if (diag && sizeof(T) == 4) {
    out[tid] = tile[tid / LB][tid % LB];  // row-major
  } else if (sizeof(T) == 8) {
    // MMA A-fragment order: (ks * 32 + lane) * 2 + h holds row g + 8h,
    // column 4 ks + t (lane = 4 g + t).
    const int ks = tid >> 6, lane = (tid >> 1) & 31, h = tid & 1;
    out[tid] = tile[(lane >> 2) + 8 * h][4 * ks + (lane & 3)];
  } else {
    out[tid] = tile[tid % LB][tid / LB];  // column-major
  }
}

template <typename T>
struct LeafArgs {
  const T *pack;  // this leaf's packed A
  int rows;       // rows of the leaf
  T *b;           // the leaf's first row (lower orientation)
  long rs_b, cs_b;
  int n;          // right-hand sides
  int *err;
  unsigned long long wait_ns;
};

template <typename T>
constexpr size_t leaf_smem() {
  return sizeof(T) * ((size_t)RING * SEG_MAX + BLK + 2 * LB * XS_LD) +
         sizeof(uint64_t) * (RING + 1) + 16;
}

// FP64: the updates are m16n8k4 .f64 MMAs, acc[q][j][e] the accumulator of
// row block warp + 8 q, columns 8 j .. 8 j + 7 (element e: row g + 8 (e >> 1),
// column 2 t + (e & 1)); panel blocks are packed in A-fragment order.
// FP32: the updates are packed FP32 FMAs (two rows per instruction), one
// lane per column, acc[q][i2] rows 2 i2 and 2 i2 + 1 of row block
// warp + 8 q; panel blocks are packed column-major, the diagonal blocks'
// inverses row-major.
template <typename T>
__global__ void __launch_bounds__(THREADS, 1) trsm_leaf_kernel(const __grid_constant__ LeafArgs<T> p) {
  constexpr bool F64 = sizeof(T) == 8;
  extern __shared__ __align__(128) unsigned char smem[];
  T *seg = (T *)smem;                 // [RING][SEG_MAX]
  T *diag0 = seg + RING * SEG_MAX;    // [BLK]
  T *xs = diag0 + BLK;                // [2][LB][XS_LD]
  uint64_t *bar = (uint64_t *)(xs + 2 * LB * XS_LD);  // RING segments + diagonal block 0
  volatile int *abort_flag = (volatile int *)(bar + RING + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int nb = (p.rows + LB - 1) / LB;
  const long col0 = (long)blockIdx.x * NBC;
  // Coalesced 16 x 32 block transfers between B and shared memory: element
  // (r, c) of pass e is taken with the stored matrix's unit stride across
  // the warp.
  const bool rows_fast = labs(p.rs_b) <= labs(p.cs_b);
  auto rc_of = [&](int e, int &r, int &c) {
    const int idx = e * 32 + lane;
    r = rows_fast ? idx % LB : idx / NBC;
    c = rows_fast ? idx / LB : idx % NBC;
  };

  if (tid == 0) {
    for (int i = 0; i <= RING; ++i) tc::mbar_init(&bar[i], 1);
    *abort_flag = 0;
    tc::fence_barrier_init();
  }
  __syncthreads();

  int issued = 0;  // segments issued (thread 0)
  auto issue = [&](int d) {
    const uint32_t bytes = (uint32_t)((nb - d) * BLK * sizeof(T));
    tc::mbar_arrive_expect_tx(&bar[d % RING], bytes);
    tc::bulk_load_1d(seg + (d % RING) * SEG_MAX, p.pack + seg_off(d, nb), bytes, &bar[d % RING]);
    issued = d + 1;
  };
  if (tid == 0) {
    tc::mbar_arrive_expect_tx(&bar[RING], BLK * sizeof(T));
    tc::bulk_load_1d(diag0, p.pack, BLK * sizeof(T), &bar[RING]);
    for (int d = 0; d < RING - 1 && d < nb - 1; ++d) issue(d);
  }

  // The CTA's 512 x 32 block of B, staged through ring slot RING - 1 (not
  // filled before the first step): warp w owns row blocks w, w + 8, w + 16,
  // w + 24.
  using Acc = typename std::conditional<F64, double[4][4][4], float2[4][8]>::type;
  Acc acc;
  {
    T *stage = seg + (RING - 1) * SEG_MAX + warp * LB * XS_LD;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int rb = warp + 8 * q;
#pragma unroll
      for (int e = 0; e < LB; ++e) {
        int r, c;
        rc_of(e, r, c);
        const int row = rb * LB + r;
        const long col = col0 + c;
        stage[r * XS_LD + c] = row < p.rows && col < p.n ? p.b[row * p.rs_b + col * p.cs_b] : T(0);
      }
      __syncwarp();
      if constexpr (F64) {
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e)
            acc[q][j][e] = stage[(g + 8 * (e >> 1)) * XS_LD + 8 * j + 2 * t + (e & 1)];
      } else {
#pragma unroll
        for (int i2 = 0; i2 < 8; ++i2)
          acc[q][i2] = make_float2(stage[(2 * i2) * XS_LD + lane], stage[(2 * i2 + 1) * XS_LD + lane]);
      }
      __syncwarp();
    }
  }
  // The staging slot is free (and its generic-proxy writes ordered before
  // the bulk copy that refills it) before any copy targets it.
  tc::fence_proxy_async();
  __syncthreads();

  // Owner of a block (warp blk % 8, accumulators acc[q] with q = blk / 8,
  // fully updated): X = inv(D) R with the packed inverse of its diagonal
  // block, into xout (row-major, XS_LD) for the other warps' updates.
  auto solve = [&](int q, const T *dinv, T *xout) {
    if constexpr (F64) {
      // R (accumulator layout) -> xout -> B fragments; X = inv(D) R as
      // 4 x 4 m16n8k4 MMAs (A = inv(D) in fragment order), accumulated in
      // the now free acc[q]; X -> xout.
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
          xout[(g + 8 * (e >> 1)) * XS_LD + 8 * j + 2 * t + (e & 1)] = acc[q][j][e];
      __syncwarp();
      double r[4][4];
#pragma unroll
      for (int ks = 0; ks < 4; ++ks)
#pragma unroll
        for (int j = 0; j < 4; ++j) r[ks][j] = xout[(4 * ks + t) * XS_LD + 8 * j + g];
      __syncwarp();
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[q][j][e] = 0.0;
      const double2 *af = (const double2 *)dinv;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        const double2 a = af[ks * 32 + lane];
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[q][j], a.x, a.y, r[ks][j]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e)
          xout[(g + 8 * (e >> 1)) * XS_LD + 8 * j + 2 * t + (e & 1)] = acc[q][j][e];
    } else {
      // One lane per column: x_i = sum_{p <= i} inv(D)_ip r_p (16 independent
      // dot products over broadcast rows of the row-major inverse).
      float r[LB];
#pragma unroll
      for (int i2 = 0; i2 < 8; ++i2) {
        r[2 * i2] = acc[q][i2].x;
        r[2 * i2 + 1] = acc[q][i2].y;
      }
#pragma unroll
      for (int i = 0; i < LB; ++i) {
        const float4 *row = (const float4 *)(dinv + i * LB);
        float x = 0.f;
#pragma unroll
        for (int v = 0; v <= i / 4; ++v) {
          const float4 w = row[v];
          x = fmaf(w.x, r[4 * v], x);
          if (4 * v + 1 <= i) x = fmaf(w.y, r[4 * v + 1], x);
          if (4 * v + 2 <= i) x = fmaf(w.z, r[4 * v + 2], x);
          if (4 * v + 3 <= i) x = fmaf(w.w, r[4 * v + 3], x);
        }
        xout[i * XS_LD + lane] = x;
      }
    }
    __syncwarp();
  };

  // Solved block blk (in xsrc) -> B, by all 256 threads, coalesced along the
  // stored matrix's unit stride.
  auto write_block = [&](int blk, const T *xsrc) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int idx = tid + h * THREADS;
      const int r = rows_fast ? idx % LB : idx / NBC, c = rows_fast ? idx / LB : idx % NBC;
      const int row = blk * LB + r;
      const long col = col0 + c;
      if (row < p.rows && col < p.n) p.b[row * p.rs_b + col * p.cs_b] = xsrc[r * XS_LD + c];
    }
  };

  // acc[q] -= A_rb,d X_d for row blocks rb = warp + 8 q, q = Q0 .. 3, all in
  // one unrolled sequence so that the blocks' independent MMA / FMA chains
  // interleave; X_d's operand fragments (xb / xr) are loaded once per step.
  // Row blocks past the leaf (rb >= nb) multiply a zero block instead of
  // reading past the segment.
  using XFrag = typename std::conditional<F64, double[4][4], float[LB]>::type;
  auto update_from = [&](auto q0c, const T *sg, int d, const XFrag &xf) {
    constexpr int Q0 = decltype(q0c)::value;
    if constexpr (F64) {
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        double2 a[4];
#pragma unroll
        for (int q = Q0; q < 4; ++q) {
          const int rb = warp + 8 * q;
          a[q] = rb < nb ? ((const double2 *)(sg + (rb - d - 1) * BLK))[ks * 32 + lane]
                         : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int q = Q0; q < 4; ++q)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma(acc[q][j], -a[q].x, -a[q].y, xf[ks][j]);
      }
    } else {
#pragma unroll
      for (int kk = 0; kk < LB; ++kk) {
        const float xv = xf[kk];
#pragma unroll
        for (int q = Q0; q < 4; ++q) {
          const int rb = warp + 8 * q;
          if (rb >= nb) continue;
          const float4 *col = (const float4 *)(sg + (rb - d - 1) * BLK + kk * LB);
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            const float4 a = col[v];
            acc[q][2 * v] =
                __ffma2_rn(make_float2(a.x, a.y), make_float2(xv, xv), acc[q][2 * v]);
            acc[q][2 * v + 1] =
                __ffma2_rn(make_float2(a.z, a.w), make_float2(xv, xv), acc[q][2 * v + 1]);
          }
        }
      }
    }
  };
  // The owner's block d + 1 alone (block 0 of the segment).
  auto update_one = [&](int q, const T *sg, const XFrag &xf) {
    if constexpr (F64) {
      const double2 *af = (const double2 *)sg;
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        const double2 a = af[ks * 32 + lane];
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[q][j], -a.x, -a.y, xf[ks][j]);
      }
    } else {
#pragma unroll
      for (int kk = 0; kk < LB; ++kk) {
        const float xv = xf[kk];
        const float4 *col = (const float4 *)(sg + kk * LB);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const float4 a = col[v];
          acc[q][2 * v] = __ffma2_rn(make_float2(a.x, a.y), make_float2(xv, xv), acc[q][2 * v]);
          acc[q][2 * v + 1] =
              __ffma2_rn(make_float2(a.z, a.w), make_float2(xv, xv), acc[q][2 * v + 1]);
        }
      }
    }
  };

  int d = 0;
  bool ok = tc::mbar_wait(&bar[RING], 0, abort_flag, p.err, p.wait_ns);
  if (__syncthreads_and(ok)) {
    if (warp == 0) solve(0, diag0, xs);
    for (; d + 1 < nb; ++d) {
      ok = tc::mbar_wait(&bar[d % RING], (d / RING) & 1, abort_flag, p.err, p.wait_ns);
      // X_d is in xs[d & 1], segment d has landed, and every warp is done
      // with step d - 1 (so its ring slot, (d + 2) % RING, is free).
      if (!__syncthreads_and(ok)) break;
      if (tid == 0 && d + 2 <= nb - 2) issue(d + 2);
      const T *sg = seg + (d % RING) * SEG_MAX;
      const T *xd = xs + (d & 1) * LB * XS_LD;
      XFrag xf;
      if constexpr (F64) {
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)
#pragma unroll
          for (int j = 0; j < 4; ++j) xf[ks][j] = xd[(4 * ks + t) * XS_LD + 8 * j + g];
      } else {
#pragma unroll
        for (int kk = 0; kk < LB; ++kk) xf[kk] = -xd[kk * XS_LD + lane];
      }
      // (q runs over compile-time values so the accumulators stay in
      // registers.)  The owner of block d + 1 goes first: its update and
      // solve are the step's critical path.
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int rb = warp + 8 * q;
        if (rb == d + 1) {
          update_one(q, sg, xf);
          solve(q, sg + (nb - 1 - d) * BLK, xs + ((d + 1) & 1) * LB * XS_LD);
        }
      }
      write_block(d, xd);
      // This warp's blocks below d + 1: q >= qlo.
      const int qlo = d + 1 - warp < 0 ? 0 : (d + 1 - warp) / 8 + 1;
      switch (qlo) {
        case 0: update_from(std::integral_constant<int, 0>(), sg, d, xf); break;
        case 1: update_from(std::integral_constant<int, 1>(), sg, d, xf); break;
        case 2: update_from(std::integral_constant<int, 2>(), sg, d, xf); break;
        case 3: update_from(std::integral_constant<int, 3>(), sg, d, xf); break;
        default: break;
      }
    }
    if (d + 1 == nb) {
      __syncthreads();  // the last block, solved in the last step
      write_block(d, xs + (d & 1) * LB * XS_LD);
    }
  } else {
    d = -1;  // diagonal block 0 never arrived
  }
  if (d + 1 < nb && tid == 0) {
    // Gave up: wait (bounded) for this CTA's copies still in flight.
    if (d < 0) tc::mbar_wait_drain(&bar[RING], 0);
    for (int s = d < 0 ? 0 : d; s < issued; ++s) tc::mbar_wait_drain(&bar[s % RING], (s / RING) & 1);
  }
}

}  // namespace

extern "C" long b200_trsm_leaf_rows(void) { return (long)LB * LEAF_BLOCKS; }

extern "C" long b200_trsm_leaf_stride(void) {
  return (long)BLK * LEAF_BLOCKS * (LEAF_BLOCKS + 1) / 2;
}

// Packs every leaf of op(A) (order m, normalised to lower / upper with
// strides) for trsm_leaf_kernel: leaves * b200_trsm_leaf_stride() elements.
extern "C" int b200_trsm_leaf_pack(int dtype, const void *a, long rs_a, long cs_a, int m,
                                   int lower, int unit, void *out) {
  if (m <= 0) return B200_OK;
  cudaStream_t s = b200_cur_stream();
  const long L = b200_trsm_leaf_rows();
  const long leaves = b200_ceil_div(m, L);
  if (leaves * LEAF_BLOCKS > 65535) return b200_set_error(B200_EINVAL, "trsm: order too large");
  LeafPackArgs pa{a, rs_a, cs_a, m, (int)L, lower, unit, out, b200_trsm_leaf_stride()};
  dim3 grid(LEAF_BLOCKS, (unsigned)(leaves * LEAF_BLOCKS));
  B200ProfScope prof(dtype == B200_F32 ? "trsm_leaf_pack_s" : "trsm_leaf_pack_d", s);
  if (dtype == B200_F32) trsm_leaf_pack_kernel<float><<<grid, 256, 0, s>>>(pa);
  else trsm_leaf_pack_kernel<double><<<grid, 256, 0, s>>>(pa);
  B200_LAUNCH_CHECK();
  return B200_OK;
}

// Solves one leaf (`rows` rows) of a packed solve for n right-hand sides:
// b points at the leaf's first row in lower orientation (for an upper leaf,
// its last row, with rs_b negated).
template <typename T>
int leaf_solve(const void *pack, int rows, T *b, long rs_b, long cs_b, int n) {
  if (rows <= 0 || n <= 0) return B200_OK;
  cudaStream_t s = b200_cur_stream();
  static std::once_flag once;
  static int conf = B200_OK;
  constexpr size_t smem = leaf_smem<T>();
  B200_TRY(b200_once(once, conf, "trsm leaf kernel: set-up failed", []() -> int {
    B200_CUDA_TRY(cudaFuncSetAttribute(trsm_leaf_kernel<T>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return B200_OK;
  }));
  LeafArgs<T> la{(const T *)pack, rows, b, rs_b, cs_b, n, b200_device_error_word(), B200_WAIT_NS};
  const long grid = b200_ceil_div(n, NBC);
  if (grid > 0x7fffffffL) return b200_set_error(B200_EINVAL, "trsm: too many right-hand sides");
  B200ProfScope prof(sizeof(T) == 4 ? "trsm_leaf_s" : "trsm_leaf_d", s);
  trsm_leaf_kernel<T><<<(unsigned)grid, THREADS, smem, s>>>(la);
  B200_LAUNCH_CHECK();
  return B200_OK;
}

extern "C" int b200_trsm_leaf_solve(int dtype, const void *pack, int rows, void *b, long rs_b,
                                    long cs_b, int n) {
  if (dtype == B200_F32) return leaf_solve<float>(pack, rows, (float *)b, rs_b, cs_b, n);
  return leaf_solve<double>(pack, rows, (double *)b, rs_b, cs_b, n);
}
