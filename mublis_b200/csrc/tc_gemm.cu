// tc_gemm.cu -- tcgen05 forms of the L3 contraction.
//
// BF16x3 / BF16x6 (FP32-class):  every FP32 operand element x is split in
// the pack pass into bf16 terms x = h + l (+ l2); the kernel accumulates in
// one FP32 TMEM accumulator the products whose term indices sum to < TERMS
// (hi*hi + hi*lo + lo*hi for x3; plus hi*lo2 + lo*lo + lo2*hi for x6).
//
// Kernel shape (sm_100a, one CTA per SM, persistent over output tiles):
//   warp 0      TMA producer: per k-block, TERMS A-plane tiles (128 x 32 bf16)
//               and TERMS B-plane tiles (256 x 32 bf16), 64-byte swizzle,
//               into a STAGES-deep ring guarded by full/empty mbarriers
//   warp 1      MMA issuer: one thread issues tcgen05.mma (M=128, N=256,
//               K=16) into a TMEM accumulator, commits stage releases
//   warp 2      allocates / frees 512 TMEM columns: two 256-column window
//               accumulators, so the MMAs of window w+1 overlap the drain
//               of window w
//   warps 4-11  epilogue (two warps per TMEM lane quadrant, 128 columns
//               each): every FLUSH k-blocks (256 k) a thread folds its row's
//               window accumulator (tcgen05.ld) into a 128-wide FP32 running
//               sum held in registers, with round-to-nearest adds; after the
//               last window it applies alpha/beta, the domain's ji mask and
//               the m/n edge and stores column-major C with coalesced writes
// Why windows: the tensor core's FP32 accumulation does not round to
// nearest, so its error grows with the number of accumulation steps; with
// a 256-deep window the sum over windows is an ordinary RN FP32 sum and the
// error matches a scalar FP32 loop.
// The tile walk, domain pruning and k-range clipping are the same as the
// plain kernel's (gemm_simt.cu), i.e. the reference driver's
// (frame/l3/l3_driver.c:130-171); a tile without update writes beta * C.
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>

#include "kernels.cuh"
#include "tc_common.cuh"
#include "tc_gemm.cuh"

// ---- host helpers ------------------------------------------------------------

namespace {

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;
int *g_err_host = nullptr;
int *g_err_dev = nullptr;
std::once_flag g_err_once;

void init_encode() {
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
          cudaSuccess &&
      q == cudaDriverEntryPointSuccess)
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
}

void init_err() {
  if (cudaHostAlloc((void **)&g_err_host, sizeof(int), cudaHostAllocMapped) == cudaSuccess) {
    *g_err_host = 0;
    cudaHostGetDevicePointer((void **)&g_err_dev, g_err_host, 0);
  }
}

}  // namespace

int *b200_device_error_word() {
  std::call_once(g_err_once, init_err);
  return g_err_dev;
}

extern "C" int b200_take_device_error(void) {
  if (!g_err_host) return 0;
  int e = *(volatile int *)g_err_host;
  if (e) *(volatile int *)g_err_host = 0;
  return e;
}

int b200_make_tmap(CUtensorMap *map, const void *base, int is_bf16, long k, long rows, int box_k,
                   int box_rows, int swz) {
  std::call_once(g_encode_once, init_encode);
  if (!g_encode) return b200_set_error(B200_ECUDA, "cuTensorMapEncodeTiled unavailable");
  const int elt = is_bf16 ? 2 : 1;
  cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(k * elt)};
  cuuint32_t box[2] = {(cuuint32_t)box_k, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(map, is_bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8,
                        2, const_cast<void *>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE,
                        swz == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return b200_set_error(B200_ECUDA, "cuTensorMapEncodeTiled failed");
  return B200_OK;
}

int b200_make_tmap_f64(CUtensorMap *map, const void *base, long inner, long outer,
                       long outer_stride, int box_inner, int box_outer, int swizzle128) {
  std::call_once(g_encode_once, init_encode);
  if (!g_encode) return b200_set_error(B200_ECUDA, "cuTensorMapEncodeTiled unavailable");
  cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
  cuuint64_t strides[1] = {(cuuint64_t)(outer_stride * (long)sizeof(double))};
  cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void *>(base), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return b200_set_error(B200_ECUDA, "cuTensorMapEncodeTiled (f64) failed");
  return B200_OK;
}

// ---- shared tile walk ---------------------------------------------------------

namespace {

struct TileWalk {
  int tiles_m, tiles_n, bm, bn;
  int m, n, kblocks, bk;
  long k;
  int jp, ji, pi;

  __device__ __forceinline__ void coords(int idx, int &tm, int &tn) const {
    constexpr int G = 8;
    int group = idx / (G * tiles_n);
    int first = group * G;
    int gsize = min(tiles_m - first, G);
    int in_group = idx % (G * tiles_n);
    tm = first + in_group % gsize;
    tn = in_group / gsize;
  }
  __device__ __forceinline__ bool valid(int tm, int tn) const {
    long m0 = (long)tm * bm, n0 = (long)tn * bn;
    if (ji == MUBLIS_L3_LOWER && n0 >= m0 + bm) return false;
    if (ji == MUBLIS_L3_UPPER && n0 + bn <= m0) return false;
    return true;
  }
  __device__ __forceinline__ void krange(int tm, int tn, int &kb0, int &kb1) const {
    long m0 = (long)tm * bm, n0 = (long)tn * bn;
    long lo = 0, hi = k;
    if (jp == MUBLIS_L3_LOWER) lo = max(lo, n0);
    if (jp == MUBLIS_L3_UPPER) hi = min(hi, n0 + bn);
    if (pi == MUBLIS_L3_LOWER) hi = min(hi, m0 + bm);
    if (pi == MUBLIS_L3_UPPER) lo = max(lo, m0);
    kb0 = (int)(lo / bk);
    kb1 = hi > lo ? (int)((hi + bk - 1) / bk) : kb0;
  }
};

struct Bf16Params {
  TileWalk w;
  long mpad, npad;  // rows per plane
  float alpha, beta;
  float *c;
  long rs_c, cs_c;
  int *err;
  // fp16 form: bits of max |x| per row of op(A) / column of op(B); the
  // planes hold x * 2^-e, so the result is scaled back by 2^(e_i + f_j).
  const int *aexp, *bexp;  // fp16x3: row / column scale exponents
};

template <int TERMS, int STAGES>
struct Bf16Cfg {
  static constexpr int BM = 128, BN = 256, SWZ = 64, BK = SWZ / 2;
  static constexpr int A_TILE = BM * SWZ, B_TILE = BN * SWZ;
  static constexpr int STAGE_BYTES = TERMS * (A_TILE + B_TILE);
  static constexpr int KSTEPS = SWZ / 32;
  static constexpr int FLUSH = 8;  // k-blocks (8 x 32 = 256 k) per TMEM window
  static constexpr int THREADS = 384;
  static constexpr int EPI_THREADS = 256;
  static constexpr int HALF = BN / 2;  // columns per epilogue thread
  static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 + 256;
  static constexpr uint32_t TMEM_COLS = 512;
};

// Register split of the tensor-core kernels: launched at 168 registers per
// thread (384 threads), warpgroup 0 (TMA producer, MMA issuer, TMEM owner)
// drops to 56 and the two epilogue warpgroups rise to 216, which holds the
// 128 FP32 running sums per thread, four 16-column TMEM loads in flight and
// a 16-column batch of C without spilling (at one 168 budget for all
// warps, the fp16x3 epilogue spilled part of its running sums to local
// memory on every window drain).
constexpr int TC_PRODUCER_REGS = 56, TC_EPILOGUE_REGS = 216;

// True when warpgroup 0 dropping to TC_PRODUCER_REGS frees enough for the
// two epilogue warpgroups to rise to TC_EPILOGUE_REGS from the compiled
// kernel's per-thread allocation `launch_regs` (384 threads).  An increase
// that cannot be granted waits forever, so the launchers check this first.
inline bool tc_register_split_fits(int launch_regs) {
  return launch_regs >= TC_PRODUCER_REGS &&
         128L * (launch_regs - TC_PRODUCER_REGS) >= 256L * (TC_EPILOGUE_REGS - launch_regs);
}

template <int TERMS, int STAGES, bool F16 = false>
__global__ void __launch_bounds__(384, 1)
    tc_bf16_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                   Bf16Params p) {
  using C = Bf16Cfg<TERMS, STAGES>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem =
      (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(smem + STAGES * C::STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *tfull = empty + STAGES;
  uint64_t *tempty = tfull + 2;
  uint64_t *drain = tempty + 2;
  uint32_t *tmem_slot = (uint32_t *)(drain + 1);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      tc::mbar_init(&tfull[a], 1);
      tc::mbar_init(&tempty[a], C::EPI_THREADS);
    }
    tc::mbar_init(drain, 1);
    *abort_flag = 0;
    tc::fence_barrier_init();
    tc::tma_prefetch_desc(&tmA);
    tc::tma_prefetch_desc(&tmB);
  }
  if (warp == 2) tc::tmem_alloc(tmem_slot, C::TMEM_COLS);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  const TileWalk &w = p.w;
  const int num_tiles = w.tiles_m * w.tiles_n;
  auto sa = [&](int s, int t) { return smem + s * C::STAGE_BYTES + t * C::A_TILE; };
  auto sb = [&](int s, int t) {
    return smem + s * C::STAGE_BYTES + TERMS * C::A_TILE + t * C::B_TILE;
  };

  // Each warpgroup's register share is set at the top of the branch that
  // holds its role, so the compiler allocates each role's code against it.
  if (warp < 4) {
  tc::setmaxnreg_dec<TC_PRODUCER_REGS>();
  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer ----------------
    int stage = 0;
    uint32_t phase = 0;
    int issued = 0;
    bool ok = true;
    for (int idx = blockIdx.x; idx < num_tiles && ok; idx += gridDim.x) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      for (int kb = kb0; kb < kb1; ++kb) {
        if (!tc::mbar_wait(&empty[stage], phase ^ 1, abort_flag, p.err)) { ok = false; break; }
        tc::mbar_arrive_expect_tx(&full[stage], C::STAGE_BYTES);
#pragma unroll
        for (int t = 0; t < TERMS; ++t)
          tc::tma_load_2d(sa(stage, t), &tmA, &full[stage], kb * C::BK,
                          (int)(t * p.mpad + (long)tm * C::BM));
#pragma unroll
        for (int t = 0; t < TERMS; ++t)
          tc::tma_load_2d(sb(stage, t), &tmB, &full[stage], kb * C::BK,
                          (int)(t * p.npad + (long)tn * C::BN));
        ++issued;
        if (++stage == STAGES) { stage = 0; phase ^= 1; }
      }
    }
    // Drain: wait (bounded) for the loads of the last ring's worth of stages.
    int pending = issued < STAGES ? issued : STAGES;
    for (int q = 0; q < pending; ++q) {
      if (--stage < 0) { stage = STAGES - 1; phase ^= 1; }
      if (!tc::mbar_wait_drain(&full[stage], phase)) break;
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t IDESC = F16 ? tc::idesc_f16(C::BM, C::BN) : tc::idesc_bf16(C::BM, C::BN);
    int stage = 0, acc = 0;
    uint32_t phase = 0, acc_phase = 0;
    bool ok = true, any = false;
    for (int idx = blockIdx.x; idx < num_tiles && ok; idx += gridDim.x) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      for (int c0 = kb0; c0 < kb1 && ok; c0 += C::FLUSH) {
        const int c1 = min(kb1, c0 + C::FLUSH);
        // The epilogue has drained this window buffer's previous use.
        if (!tc::mbar_wait(&tempty[acc], acc_phase ^ 1, abort_flag, p.err)) { ok = false; break; }
        tc::tc_fence_after();
        const uint32_t d = tmem_base + (uint32_t)(acc * C::BN);
        for (int kb = c0; kb < c1; ++kb) {
          if (!tc::mbar_wait(&full[stage], phase, abort_flag, p.err)) { ok = false; break; }
          tc::tc_fence_after();
#pragma unroll
          for (int ks = 0; ks < C::KSTEPS; ++ks) {
            // Small terms first, the hi*hi product last.
#pragma unroll
            for (int sum = TERMS - 1; sum >= 0; --sum) {
#pragma unroll
              for (int ta = 0; ta <= sum; ++ta) {
                const int tb = sum - ta;
                uint64_t ad = tc::smem_desc(sa(stage, ta), C::SWZ) + (uint64_t)((ks * 32) >> 4);
                uint64_t bd = tc::smem_desc(sb(stage, tb), C::SWZ) + (uint64_t)((ks * 32) >> 4);
                const bool first = kb == c0 && ks == 0 && sum == TERMS - 1 && ta == 0;
                tc::mma_bf16(d, ad, bd, IDESC, first ? 0u : 1u);
              }
            }
          }
          tc::mma_commit(&empty[stage]);
          any = true;
          if (++stage == STAGES) { stage = 0; phase ^= 1; }
        }
        if (!ok) break;
        tc::mma_commit(&tfull[acc]);
        if (++acc == 2) { acc = 0; acc_phase ^= 1; }
      }
    }
    if (any) {  // every issued MMA has completed before TMEM is released
      tc::mma_commit(drain);
      tc::mbar_wait(drain, 0, abort_flag, p.err);
    }
  }
  } else {
    tc::setmaxnreg_inc<TC_EPILOGUE_REGS>();
    // ---------------- epilogue ----------------
    const int quad = warp & 3;        // TMEM lanes 32*quad .. 32*quad+31
    const int half = (warp - 4) >> 2; // columns [half*128, half*128+128)
    const int row = quad * 32 + lane;
    const uint32_t lane_base = tmem_base + ((uint32_t)(quad * 32) << 16);
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    float run[C::HALF];
    for (int idx = blockIdx.x; idx < num_tiles && ok; idx += gridDim.x) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      const long gi = (long)tm * C::BM + row;
      const bool row_ok = gi < w.m;
      const long gj0 = (long)tn * C::BN + half * C::HALF;
      if (kb0 >= kb1) {  // no update: beta * C
        if (row_ok)
          for (int j = 0; j < C::HALF; ++j) {
            const long gj = gj0 + j;
            if (gj >= w.n || !b200_rel(w.ji, gj, gi)) continue;
            float *cij = p.c + gi * p.rs_c + gj * p.cs_c;
            *cij = p.beta != 0.f ? p.beta * *cij : 0.f;
          }
        continue;
      }
      const int nwin = (kb1 - kb0 + C::FLUSH - 1) / C::FLUSH;
      float *crow = p.c + gi * p.rs_c;
      for (int win = 0; win < nwin; ++win) {
        if (win == nwin - 1 && row_ok && p.beta != 0.f) {
          // While the tile's last window is multiplied, pull the C values
          // the final store reads into L2.
#pragma unroll 8
          for (int j = 0; j < C::HALF; ++j)
            if (gj0 + j < w.n)
              asm volatile("prefetch.global.L2 [%0];" ::"l"(crow + (gj0 + j) * p.cs_c));
        }
        // Every lane observes the barrier; the outcome is made warp-uniform
        // because the TMEM loads below are .sync.aligned.
        int wok = tc::mbar_wait(&tfull[acc], acc_phase, abort_flag, p.err);
        if (!__all_sync(0xffffffffu, wok)) { ok = false; break; }
        tc::tc_fence_after();
        const uint32_t base = lane_base + (uint32_t)(acc * C::BN + half * C::HALF);
        // Four 16-column TMEM loads in flight per wait.
#pragma unroll
        for (int g0 = 0; g0 < C::HALF / 16; g0 += 4) {
          uint32_t r[4][16];
#pragma unroll
          for (int q = 0; q < 4; ++q) tc::tmem_ld16(base + (uint32_t)((g0 + q) * 16), r[q]);
          tc::tmem_wait_ld();
#pragma unroll
          for (int q = 0; q < 4; ++q) tc::tmem_tie16(r[q]);
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int c = (g0 + q) * 16 + j;
              run[c] = win == 0 ? __uint_as_float(r[q][j])
                                : __fadd_rn(run[c], __uint_as_float(r[q][j]));
            }
        }
        tc::tc_fence_before();
        tc::mbar_arrive(&tempty[acc]);
        if (++acc == 2) { acc = 0; acc_phase ^= 1; }
      }
      if (!ok) break;
      if (row_ok) {
        // In batches of 16 columns: the batch's loads (C, and the column
        // scales of fp16x3) are issued before its stores.  A load / store
        // chain per element pays one memory round trip each, and while this
        // store runs the MMAs of the next tile stall after two windows.
        const int ei = F16 ? p.aexp[gi] : 0;
#pragma unroll
        for (int j0 = 0; j0 < C::HALF; j0 += 16) {
          float cv[16];
          int sc[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const long gj = gj0 + j0 + j;
            const bool in = gj < w.n && b200_rel(w.ji, gj, gi);
            cv[j] = in && p.beta != 0.f ? crow[gj * p.cs_c] : 0.f;
            sc[j] = F16 && in ? p.bexp[gj] : 0;
          }
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const long gj = gj0 + j0 + j;
            if (gj >= w.n || !b200_rel(w.ji, gj, gi)) continue;
            float v = F16 ? p.alpha * b200_pow2_scale(run[j0 + j],
                                                      ei + sc[j] - 2 * B200_FP16_SCALE_EXP)
                          : p.alpha * run[j0 + j];
            if (p.beta != 0.f) v = fmaf(p.beta, cv[j], v);
            crow[gj * p.cs_c] = v;
          }
        }
      }
    }
  }

  tc::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem_base, C::TMEM_COLS);
  }
}

// ---- CTA-pair form ----------------------------------------------------------
//
// The same contraction with 256 x 256 tiles on a pair of SMs (a cluster of
// two CTAs, tcgen05 cta_group::2).  Each CTA TMA-loads its 128 rows of
// op(A) and its 128 rows (columns of the tile) of op(B) into its own shared
// memory, completing the bytes on the leader's (rank 0) stage barrier; the
// leader issues the M = 256, N = 256 MMAs, which read both CTAs' tiles and
// write each CTA's 128 accumulator rows into that CTA's TMEM; its commits
// arrive on the stage-free and window-ready barriers of both CTAs; each
// epilogue warp releases a window on the leader's barrier.  Per SM and MMA
// the tensor cores read 4 KB of A and 4 KB of B from shared memory instead
// of 4 KB and 8 KB, which is what bounds the three-product forms on one SM
// (operand reads plus the TMA fills exceed the shared-memory bandwidth).
// The MMA sequence per output element (k order, products, windows) is the
// single-SM kernel's.
template <int TERMS, int STAGES>
struct Bf16PairCfg {
  static constexpr int BM = 128, BN = 128, SWZ = 64, BK = SWZ / 2;  // per CTA
  static constexpr int TILE_M = 256, TILE_N = 256;                  // per pair
  static constexpr int A_TILE = BM * SWZ, B_TILE = BN * SWZ;
  static constexpr int STAGE_BYTES = TERMS * (A_TILE + B_TILE);
  static constexpr int KSTEPS = SWZ / 32;
  static constexpr int FLUSH = 8;
  static constexpr int THREADS = 384;
  static constexpr int EPI_WARPS = 8;
  static constexpr int HALF = TILE_N / 2;  // columns per epilogue thread
  static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 + 256;
  static constexpr uint32_t TMEM_COLS = 512;
};

template <int TERMS, int STAGES, bool F16 = false>
__global__ void __launch_bounds__(384, 1)
    tc_bf16_pair_kernel(const __grid_constant__ CUtensorMap tmA,
                        const __grid_constant__ CUtensorMap tmB, Bf16Params p) {
  using C = Bf16PairCfg<TERMS, STAGES>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem =
      (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(smem + STAGES * C::STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *tfull = empty + STAGES;
  uint64_t *tempty = tfull + 2;
  uint64_t *drain = tempty + 2;
  uint32_t *tmem_slot = (uint32_t *)(drain + 1);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = tc::cluster_rank();
  const bool leader = rank == 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full[s], 1);   // leader: its expect_tx; bytes of both CTAs
      tc::mbar_init(&empty[s], 1);  // the leader's commit, in both CTAs
    }
    for (int a = 0; a < 2; ++a) {
      tc::mbar_init(&tfull[a], 1);
      tc::mbar_init(&tempty[a], 2 * C::EPI_WARPS);  // leader: one arrival per epilogue warp of the pair
    }
    tc::mbar_init(drain, 1);
    *abort_flag = 0;
    tc::fence_barrier_init();
    tc::tma_prefetch_desc(&tmA);
    tc::tma_prefetch_desc(&tmB);
  }
  if (warp == 2) tc::tmem_alloc_pair(tmem_slot, C::TMEM_COLS);
  tc::tc_fence_before();
  __syncthreads();
  tc::cluster_sync();  // both CTAs' barriers initialised before any remote use
  tc::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  const TileWalk &w = p.w;  // bm = bn = 256: pair tiles
  const int num_tiles = w.tiles_m * w.tiles_n;
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  auto sa = [&](int s, int t) { return smem + s * C::STAGE_BYTES + t * C::A_TILE; };
  auto sb = [&](int s, int t) {
    return smem + s * C::STAGE_BYTES + TERMS * C::A_TILE + t * C::B_TILE;
  };

  if (warp < 4) {
  tc::setmaxnreg_dec<TC_PRODUCER_REGS>();
  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    int stage = 0;
    uint32_t phase = 0;
    int issued = 0;
    bool ok = true;
    for (int idx = pair; idx < num_tiles && ok; idx += npairs) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      const int arow = (int)((long)tm * C::TILE_M + rank * C::BM);
      const int brow = (int)((long)tn * C::TILE_N + rank * C::BN);
      for (int kb = kb0; kb < kb1; ++kb) {
        if (!tc::mbar_wait(&empty[stage], phase ^ 1, abort_flag, p.err)) { ok = false; break; }
        if (leader) tc::mbar_arrive_expect_tx(&full[stage], 2 * C::STAGE_BYTES);
        const uint32_t fb = tc::map_rank(&full[stage], 0);
#pragma unroll
        for (int t = 0; t < TERMS; ++t)
          tc::tma_load_2d_pair(sa(stage, t), &tmA, fb, kb * C::BK, (int)(t * p.mpad + arow));
#pragma unroll
        for (int t = 0; t < TERMS; ++t)
          tc::tma_load_2d_pair(sb(stage, t), &tmB, fb, kb * C::BK, (int)(t * p.npad + brow));
        ++issued;
        if (++stage == STAGES) { stage = 0; phase ^= 1; }
      }
    }
    // Drain (leader): the last ring's worth of stages has landed in both
    // CTAs (their bytes complete on the leader's barriers).
    if (leader) {
      int pending = issued < STAGES ? issued : STAGES;
      for (int q = 0; q < pending; ++q) {
        if (--stage < 0) { stage = STAGES - 1; phase ^= 1; }
        if (!tc::mbar_wait_drain(&full[stage], phase)) break;
      }
    }
  } else if (warp == 1 && lane == 0 && leader) {
    // ---------------- MMA issuer (leader) ----------------
    constexpr uint32_t IDESC = F16 ? tc::idesc_f16(C::TILE_M, C::TILE_N)
                                   : tc::idesc_bf16(C::TILE_M, C::TILE_N);
    int stage = 0, acc = 0;
    uint32_t phase = 0, acc_phase = 0;
    bool ok = true, any = false;
    for (int idx = pair; idx < num_tiles && ok; idx += npairs) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      for (int c0 = kb0; c0 < kb1 && ok; c0 += C::FLUSH) {
        const int c1 = min(kb1, c0 + C::FLUSH);
        // Both CTAs' epilogues have drained this window buffer.
        if (!tc::mbar_wait(&tempty[acc], acc_phase ^ 1, abort_flag, p.err)) { ok = false; break; }
        tc::tc_fence_after();
        const uint32_t d = tmem_base + (uint32_t)(acc * C::TILE_N);
        for (int kb = c0; kb < c1; ++kb) {
          if (!tc::mbar_wait(&full[stage], phase, abort_flag, p.err)) { ok = false; break; }
          tc::tc_fence_after();
#pragma unroll
          for (int ks = 0; ks < C::KSTEPS; ++ks) {
#pragma unroll
            for (int sum = TERMS - 1; sum >= 0; --sum) {
#pragma unroll
              for (int ta = 0; ta <= sum; ++ta) {
                const int tb = sum - ta;
                uint64_t ad = tc::smem_desc(sa(stage, ta), C::SWZ) + (uint64_t)((ks * 32) >> 4);
                uint64_t bd = tc::smem_desc(sb(stage, tb), C::SWZ) + (uint64_t)((ks * 32) >> 4);
                const bool first = kb == c0 && ks == 0 && sum == TERMS - 1 && ta == 0;
                tc::mma_f16_pair(d, ad, bd, IDESC, first ? 0u : 1u);
              }
            }
          }
          tc::mma_commit_pair(&empty[stage]);
          any = true;
          if (++stage == STAGES) { stage = 0; phase ^= 1; }
        }
        if (!ok) break;
        tc::mma_commit_pair(&tfull[acc]);
        if (++acc == 2) { acc = 0; acc_phase ^= 1; }
      }
    }
    if (any) {  // every issued MMA has completed before TMEM is released
      tc::mma_commit_pair(drain);
      tc::mbar_wait(drain, 0, abort_flag, p.err);
    }
  }
  } else {
    tc::setmaxnreg_inc<TC_EPILOGUE_REGS>();
    // ---------------- epilogue (both CTAs: this CTA's 128 rows) ----------------
    const int quad = warp & 3;
    const int half = (warp - 4) >> 2;
    const int row = quad * 32 + lane;
    const uint32_t lane_base = tmem_base + ((uint32_t)(quad * 32) << 16);
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    float run[C::HALF];
    for (int idx = pair; idx < num_tiles && ok; idx += npairs) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      const long gi = (long)tm * C::TILE_M + rank * C::BM + row;
      const bool row_ok = gi < w.m;
      const long gj0 = (long)tn * C::TILE_N + half * C::HALF;
      if (kb0 >= kb1) {  // no update: beta * C
        if (row_ok)
          for (int j = 0; j < C::HALF; ++j) {
            const long gj = gj0 + j;
            if (gj >= w.n || !b200_rel(w.ji, gj, gi)) continue;
            float *cij = p.c + gi * p.rs_c + gj * p.cs_c;
            *cij = p.beta != 0.f ? p.beta * *cij : 0.f;
          }
        continue;
      }
      const int nwin = (kb1 - kb0 + C::FLUSH - 1) / C::FLUSH;
      float *crow = p.c + gi * p.rs_c;
      for (int win = 0; win < nwin; ++win) {
        if (win == nwin - 1 && row_ok && p.beta != 0.f) {
#pragma unroll 8
          for (int j = 0; j < C::HALF; ++j)
            if (gj0 + j < w.n)
              asm volatile("prefetch.global.L2 [%0];" ::"l"(crow + (gj0 + j) * p.cs_c));
        }
        int wok = tc::mbar_wait(&tfull[acc], acc_phase, abort_flag, p.err);
        if (!__all_sync(0xffffffffu, wok)) { ok = false; break; }
        tc::tc_fence_after();
        const uint32_t base = lane_base + (uint32_t)(acc * C::TILE_N + half * C::HALF);
#pragma unroll
        for (int g0 = 0; g0 < C::HALF / 16; g0 += 4) {
          uint32_t r[4][16];
#pragma unroll
          for (int q = 0; q < 4; ++q) tc::tmem_ld16(base + (uint32_t)((g0 + q) * 16), r[q]);
          tc::tmem_wait_ld();
#pragma unroll
          for (int q = 0; q < 4; ++q) tc::tmem_tie16(r[q]);
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const int c = (g0 + q) * 16 + j;
              run[c] = win == 0 ? __uint_as_float(r[q][j])
                                : __fadd_rn(run[c], __uint_as_float(r[q][j]));
            }
        }
        tc::tc_fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive_cluster(tc::map_rank(&tempty[acc], 0));
        if (++acc == 2) { acc = 0; acc_phase ^= 1; }
      }
      if (!ok) break;
      if (row_ok) {
        const int ei = F16 ? p.aexp[gi] : 0;
#pragma unroll
        for (int j0 = 0; j0 < C::HALF; j0 += 16) {
          float cv[16];
          int sc[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const long gj = gj0 + j0 + j;
            const bool in = gj < w.n && b200_rel(w.ji, gj, gi);
            cv[j] = in && p.beta != 0.f ? crow[gj * p.cs_c] : 0.f;
            sc[j] = F16 && in ? p.bexp[gj] : 0;
          }
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const long gj = gj0 + j0 + j;
            if (gj >= w.n || !b200_rel(w.ji, gj, gi)) continue;
            float v = F16 ? p.alpha * b200_pow2_scale(run[j0 + j],
                                                      ei + sc[j] - 2 * B200_FP16_SCALE_EXP)
                          : p.alpha * run[j0 + j];
            if (p.beta != 0.f) v = fmaf(p.beta, cv[j], v);
            crow[gj * p.cs_c] = v;
          }
        }
      }
    }
  }

  // Both CTAs: every MMA has completed (the leader's issuer waited on the
  // drain commit), every remote arrival has landed and no TMEM load is
  // pending before the pair frees its TMEM.
  tc::tc_fence_before();
  __syncthreads();
  tc::cluster_sync();
  if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc_pair(tmem_base, C::TMEM_COLS);
  }
}

template <int TERMS, int STAGES, bool F16 = false>
int launch_bf16_pair(const CUtensorMap &ta, const CUtensorMap &tb, const Bf16Params &p,
                     cudaStream_t s) {
  using C = Bf16PairCfg<TERMS, STAGES>;
  auto kern = tc_bf16_pair_kernel<TERMS, STAGES, F16>;
  static std::once_flag once;
  static int conf = B200_OK, max_clusters = 0;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(C::THREADS);
  cfg.dynamicSmemBytes = C::SMEM;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  B200_TRY(b200_once(once, conf, "bf16 pair kernel: set-up failed", [&]() -> int {
    B200_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
    cudaFuncAttributes fa;
    B200_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    if (C::THREADS != 384 || !tc_register_split_fits(fa.numRegs))
      return b200_set_error(B200_EINVAL, "bf16 pair kernel: register split does not fit its launch");
    cudaLaunchConfig_t q = cfg;
    q.gridDim = dim3(2 * b200_sm_count());
    if (cudaOccupancyMaxActiveClusters(&max_clusters, (void *)kern, &q) != cudaSuccess ||
        max_clusters < 1) {
      cudaGetLastError();
      return b200_set_error(B200_ECUDA, "bf16 pair kernel: no CTA pair can be resident");
    }
    return B200_OK;
  }));
  const int tiles = p.w.tiles_m * p.w.tiles_n;
  const int pairs = tiles < max_clusters ? tiles : max_clusters;
  cfg.gridDim = dim3(2 * pairs);
  B200ProfScope prof(F16 ? "tc_fp16x3" : (TERMS == 2 ? "tc_bf16x3" : "tc_bf16x6"), s);
  B200_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, ta, tb, p));
  return B200_OK;
}

template <int TERMS, int STAGES, bool F16 = false>
int launch_bf16(const CUtensorMap &ta, const CUtensorMap &tb, const Bf16Params &p,
                cudaStream_t s) {
  using C = Bf16Cfg<TERMS, STAGES>;
  auto kern = tc_bf16_kernel<TERMS, STAGES, F16>;
  static std::once_flag once;
  static int conf = B200_OK;
  B200_TRY(b200_once(once, conf, "bf16 kernel: set-up failed", [&]() -> int {
    B200_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
    // The warpgroup register split assumes this launch allocation; with
    // fewer registers per thread the epilogue's increase could never be
    // granted, so refuse to launch rather than wait.
    cudaFuncAttributes fa;
    B200_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    if (C::THREADS != 384 || !tc_register_split_fits(fa.numRegs))
      return b200_set_error(B200_EINVAL, "bf16 kernel: register split does not fit its launch");
    return B200_OK;
  }));
  const int sms = b200_sm_count();
  int tiles = p.w.tiles_m * p.w.tiles_n;
  int grid = tiles < sms ? tiles : sms;
  B200ProfScope prof(F16 ? "tc_fp16x3" : (TERMS == 2 ? "tc_bf16x3" : "tc_bf16x6"), s);
  kern<<<grid, C::THREADS, C::SMEM, s>>>(ta, tb, p);
  B200_LAUNCH_CHECK();
  return B200_OK;
}

}  // namespace

// Packs the FP32 operands into TERMS bf16 planes (K-major, padded) and runs
// the tcgen05 kernel.  The fp16x3 form (Ootomo and Yokota's FP16 split with
// per-row / per-column power-of-two scaling) scales row i of op(A) by
// 2^(15 - e_i) and column j of op(B) by 2^(15 - f_j) so that |x| < 2^15,
// splits into fp16 hi = rn(x) and lo = rn(x - hi) (11 + 11 significant
// bits, both normal fp16 for elements down to 2^-18 of the maximum), runs
// the same three products as bf16x3 (hi hi + hi lo + lo hi, FP32
// accumulation drained every 256 k) and scales each result by
// 2^(e_i + f_j - 30).
int tc_run_bf16(const b200_l3_desc_t *d, int form) {
  if (d->dtype != B200_F32) return b200_set_error(B200_EINVAL, "bf16 forms are FP32-only");
  const bool f16 = form == B200_FORM_FP16X3;
  const int terms = form == B200_FORM_BF16X6 ? 3 : 2;
  // 256 x 256 tiles on CTA pairs (tc_bf16_pair_kernel) from 256 rows and
  // columns on; MUBLIS_B200_TC_PAIR=0 keeps the single-SM kernel.
  static const bool pair_on = [] {
    const char *e = getenv("MUBLIS_B200_TC_PAIR");
    return !(e && !strcmp(e, "0"));
  }();
  const bool pair = pair_on && d->m >= 256 && d->n >= 256;
  const int BM = pair ? 256 : 128, BN = 256, BK = 32;
  cudaStream_t s = b200_cur_stream();
  const long ktot = (long)d->k * d->npairs;
  const long mpad = b200_round_up(d->m, BM), npad = b200_round_up(d->n, BN);
  const long kpad = b200_round_up(ktot, BK);
  if (terms * (mpad > npad ? mpad : npad) > 0x7fffffffL)
    return b200_set_error(B200_EINVAL, "bf16 form: operand too large for 32-bit TMA rows");
  void *ap = nullptr, *bp = nullptr, *amax = nullptr;
  B200_TRY(b200_alloc(&ap, sizeof(uint16_t) * terms * mpad * kpad));
  int st = b200_alloc(&bp, sizeof(uint16_t) * terms * npad * kpad);
  const mublis_l3_product_t &pr = d->product;
  PackView va[2], vb[2];
  for (int t = 0; t < d->npairs; ++t) {
    va[t] = PackView{d->a[t], d->rs_a[t], d->cs_a[t], (int)pr.a.struc, (int)pr.a.uplo,
                     (int)pr.a.diag, (int)pr.domain.pi};
    vb[t] = PackView{d->b[t], d->rs_b[t], d->cs_b[t], (int)pr.b.struc, (int)pr.b.uplo,
                     (int)pr.b.diag, (int)pr.domain.jp};
  }
  unsigned long long *am = nullptr, *bm = nullptr;
  int *ae = nullptr;
  if (f16 && st == B200_OK) {  // scales over the whole (concatenated) k
    st = b200_alloc(&amax, (sizeof(unsigned long long) + sizeof(int)) * (mpad + npad));
    am = (unsigned long long *)amax;
    bm = am + mpad;
    ae = (int *)(am + mpad + npad);
    if (st == B200_OK &&
        cudaMemsetAsync(amax, 0, sizeof(unsigned long long) * (mpad + npad), s) != cudaSuccess)
      st = b200_set_error(B200_ECUDA, "memset failed");
    for (int t = 0; t < d->npairs && st == B200_OK; ++t) {
      st = launch_absmax<float>(va[t], false, d->m, d->k, am, s);
      if (st == B200_OK) st = launch_absmax<float>(vb[t], true, d->n, d->k, bm, s);
    }
    if (st == B200_OK) st = launch_scale_exps(am, ae, mpad + npad, s);
  }
  const int xform = f16 ? PACK_FP16_SPLIT : PACK_BF16_SPLIT;
  for (int t = 0; t < d->npairs && st == B200_OK; ++t) {
    long kk0 = (long)t * d->k, kk1 = t + 1 == d->npairs ? kpad : kk0 + d->k;
    PackOut oa{ap, kpad, mpad * kpad, PACK_K_MAJOR, xform, terms, am};
    PackOut ob{bp, kpad, npad * kpad, PACK_K_MAJOR, xform, terms, bm};
    st = launch_pack<float>(va[t], false, d->m, d->k, mpad, kk0, kk1, oa, s);
    if (st == B200_OK) st = launch_pack<float>(vb[t], true, d->n, d->k, npad, kk0, kk1, ob, s);
  }
  CUtensorMap ta, tb;
  // Boxes of one CTA's tile: 128 rows of A (both forms), 256 or 128 of B.
  if (st == B200_OK) st = b200_make_tmap(&ta, ap, 1, kpad, terms * mpad, BK, 128, 64);
  if (st == B200_OK) st = b200_make_tmap(&tb, bp, 1, kpad, terms * npad, BK, pair ? 128 : BN, 64);
  if (st == B200_OK) {
    Bf16Params p;
    p.w.tiles_m = (int)(mpad / BM);
    p.w.tiles_n = (int)(npad / BN);
    p.w.bm = BM;
    p.w.bn = BN;
    p.w.m = d->m;
    p.w.n = d->n;
    p.w.k = ktot;
    p.w.bk = BK;
    p.w.kblocks = (int)(kpad / BK);
    p.w.jp = pr.domain.jp;
    p.w.ji = pr.domain.ji;
    p.w.pi = pr.domain.pi;
    p.mpad = mpad;
    p.npad = npad;
    p.alpha = (float)d->alpha;
    p.beta = (float)d->beta;
    p.c = (float *)d->c;
    p.rs_c = d->rs_c;
    p.cs_c = d->cs_c;
    p.err = b200_device_error_word();
    p.aexp = ae;
    p.bexp = ae ? ae + mpad : nullptr;
    if (pair)
      st = f16 ? launch_bf16_pair<2, 6, true>(ta, tb, p, s)
               : (terms == 2 ? launch_bf16_pair<2, 6>(ta, tb, p, s)
                             : launch_bf16_pair<3, 4>(ta, tb, p, s));
    else
      st = f16 ? launch_bf16<2, 4, true>(ta, tb, p, s)
               : (terms == 2 ? launch_bf16<2, 4>(ta, tb, p, s) : launch_bf16<3, 3>(ta, tb, p, s));
  }
  b200_free(ap);
  b200_free(bp);
  b200_free(amax);
  return st;
}

// ---- Ozaki split-integer FP64 ---------------------------------------------------
//
// Two forms share one persistent kernel (template MOD).
//
// Slices (MOD = false; Ozaki, Ogita, Oishi, Rump 2012, with the integer-MMA
// formulation of Mukunoki et al. and Uchino et al.).  op(A) row i is scaled
// by 2^-e_i and op(B) column j by 2^-f_j (e, f from the abs-max, so scaled
// values lie in (-1, 1)), and each scaled value is cut into s signed 7-bit
// slices: a = 2^e_i sum_t A_t 2^-7t, b = 2^f_j sum_u B_u 2^-7u (pack.cu).
// Then C = 2^(e_i + f_j) sum_d 2^-7d S_d with S_d = sum_{t+u=d} A_t B_u,
// keeping the diagonals d <= s + 1.  Every S_d is an exact int32 tcgen05
// (kind::i8) accumulation as long as s * kchunk * 127^2 < 2^31, so k is
// processed in chunks of 8192 and s <= 12.  The epilogue drains S_d from
// TMEM, adds ldexp(S_d, -7d) in FP64 into a per-CTA tile workspace
// (L2-resident), and on the last phase writes C = alpha * ldexp(W, e_i +
// f_j) + beta * C.  Phases (k-chunk, d) run from the smallest d
// contribution to the largest.
//
// Moduli (MOD = true; Ozaki scheme II, Ozaki, Uchino and Imamura 2025).
// op(A) row i becomes the integer row A'_i = rint(a_i * 2^(pa - e_i)) and
// op(B) column j becomes B'_j = rint(b_j * 2^(pb - f_j)), so |A'|, |B'| are
// at most 2^pa, 2^pb.  For N pairwise coprime moduli m_l <= 256 with
// product M, pa + pb is chosen so that k 2^(pa+pb) < M/2 (1 - 2^-30): the
// integer product C' = A'B' is then fixed by its residues modulo every m_l.
// Each residue plane A'_l = A' mod m_l (int8, symmetric) is packed once, and
// one int8 GEMM per modulus gives C'_l = A'_l B'_l exactly in int32 (k in
// chunks of 32768 keeps |C'_l| <= 2^29).  The epilogue reduces C'_l mod m_l
// into a byte per element of a per-CTA residue workspace; after the tile's
// last modulus it reconstructs C' by the Chinese remainder theorem,
// C' = sum_l r_l W_l - q M with W_l = (M/m_l) ((M/m_l)^-1 mod m_l) and
// q = round(sum / M), and writes C = alpha 2^(e_i + f_j - pa - pb) C' +
// beta C.  The CRT sum is exact in FP64: W_l and M are cut at bits 42 and 84
// into three 42-bit levels, each level's sum of N products r_l W_l,lev
// stays below 2^53 units of that level, and the top level minus q M_0 is
// exact as well.  N int8 GEMMs (16 give ~55-bit inputs) replace the
// s(s+1)/2 of the slice form.
//
// Tile: 256 x 256 per CTA, issued as two M=128 tcgen05 MMAs that share the
// B tile, so every byte brought into shared memory feeds 1.5x the int8
// products of a 128 x 256 tile (the int8 pipe outruns the L2 -> shared
// memory feed otherwise).  The two accumulators fill all 512 TMEM columns;
// the MMA issuer waits for the epilogue's drain at each phase boundary.

namespace {

constexpr int OZ_MAX_SLICES = 12;
constexpr int OZ_KCHUNK = 8192;    // k per exact int32 chunk, slice form
constexpr int OZ2_KCHUNK = 32768;  // k per exact int32 chunk, moduli (|C'_l| <= 2^29)

// CRT reconstruction constants of the modular form (host-computed).
struct OzCrt {
  double w[B200_MAX_MODULI][3];  // W_l cut into 42-bit levels at bits 84 / 42 / 0
  double mlev[3];                // M cut the same way
  double inv_m;                  // 1 / M
  int m[B200_MAX_MODULI], bias[B200_MAX_MODULI];
  unsigned mg[B200_MAX_MODULI];
  int bits;                      // pa + pb
};

struct OzParams {
  TileWalk w;
  long mpad, npad;
  int slices;  // slice count, or modulus count N of the modular form
  double alpha, beta;
  void *c;  // double (both forms) or float (modular form)
  long rs_c, cs_c;
  void *work;  // slices: gridDim.x tiles of 256 x 256 doubles;
               // moduli: gridDim.x x N x 256 x 256 residue bytes
  const int *aexp, *bexp;  // row / column scale exponents
  int *err;
  OzCrt crt;
};

// Three 64 KB stages of k-blocks of 128 bytes (128-byte swizzle).  Six
// stages of 32 KB (64-byte k-blocks) were measured 5% slower at 8192^3.
struct OzCfg {
  static constexpr int BM = 256, BN = 256, SWZ = 128, BK = 128, STAGES = 3;
  static constexpr int HALF_ROWS = 128;
  static constexpr int A_TILE = BM * SWZ, B_TILE = BN * SWZ;
  static constexpr int STAGE_BYTES = A_TILE + B_TILE;
  static constexpr int KSTEPS = SWZ / 32;
  static constexpr int THREADS = 384, EPI_THREADS = 256;
  static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 + 256;
  static constexpr uint32_t TMEM_COLS = 512;
};

// Phases of one k-chunk and the (t, u) plane pairs of each phase.  Slices:
// phase ph is diagonal d = s + 1 - ph with t = max(1, d - s) .. min(s, d - 1),
// u = d - t.  Moduli: phase l is the single pair (l + 1, l + 1).
template <bool MOD>
__device__ __forceinline__ void oz_pairs(int S, int ph, int &t0, int &t1, int &d) {
  if (MOD) {
    t0 = t1 = ph + 1;
    d = 2 * (ph + 1);
  } else {
    d = S + 1 - ph;
    t0 = max(1, d - S);
    t1 = min(S, d - 1);
  }
}

// CRT of one element from its N residues (the modular form's last step).
__device__ __forceinline__ double oz_crt(const OzCrt &k, double s0, double s1, double s2) {
  // All three levels enter q: with few moduli (M below 2^84) the low levels
  // carry most of the sum.  |S/M| < 2^11 and the argument's error is below
  // 2^-40, while the pa + pb margin keeps S/M at least 2^-21 away from a
  // half-integer, so q is exact.
  const double q = rint(fma(s0, k.inv_m, fma(s1, k.inv_m, s2 * k.inv_m)));
  const double t0 = fma(-q, k.mlev[0], s0);  // exact: |t0| < 2^126, a multiple of 2^84
  const double t1 = fma(-q, k.mlev[1], s1);
  const double t2 = fma(-q, k.mlev[2], s2);
  return (t0 + t1) + t2;
}

template <bool MOD, typename TC>
__global__ void __launch_bounds__(384, 1)
    tc_ozaki_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    const __grid_constant__ OzParams p) {
  using C = OzCfg;
  constexpr int STAGES = C::STAGES;
  constexpr int KCHUNK = (MOD ? OZ2_KCHUNK : OZ_KCHUNK) / C::BK;  // in k-blocks
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem =
      (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(smem + STAGES * C::STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *tfull = empty + STAGES;
  uint64_t *tempty = tfull + 1;
  uint64_t *drain = tempty + 1;
  uint32_t *tmem_slot = (uint32_t *)(drain + 1);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(tfull, 1);
    tc::mbar_init(tempty, C::EPI_THREADS);
    tc::mbar_init(drain, 1);
    *abort_flag = 0;
    tc::fence_barrier_init();
    tc::tma_prefetch_desc(&tmA);
    tc::tma_prefetch_desc(&tmB);
  }
  if (warp == 2) tc::tmem_alloc(tmem_slot, C::TMEM_COLS);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  const TileWalk &w = p.w;
  const int S = p.slices;
  const int num_tiles = w.tiles_m * w.tiles_n;
  auto sa = [&](int st) { return smem + st * C::STAGE_BYTES; };
  auto sb = [&](int st) { return smem + st * C::STAGE_BYTES + C::A_TILE; };

  // Register shares per warpgroup, set where each role begins (as in the
  // BF16 kernel): the epilogue keeps four 16-column TMEM loads in flight.
  if (warp < 4) {
  tc::setmaxnreg_dec<TC_PRODUCER_REGS>();
  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer ----------------
    int stage = 0, issued = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (int idx = blockIdx.x; idx < num_tiles && ok; idx += gridDim.x) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      for (int c0 = kb0; c0 < kb1 && ok; c0 += KCHUNK) {
        const int c1 = min(kb1, c0 + KCHUNK);
        for (int ph = 0; ph < S && ok; ++ph) {
          int t0, t1, d;
          oz_pairs<MOD>(S, ph, t0, t1, d);
          for (int t = t0; t <= t1 && ok; ++t) {
            const int u = d - t;
            for (int kb = c0; kb < c1; ++kb) {
              if (!tc::mbar_wait(&empty[stage], phase ^ 1, abort_flag, p.err)) { ok = false; break; }
              tc::mbar_arrive_expect_tx(&full[stage], C::STAGE_BYTES);
              tc::tma_load_2d(sa(stage), &tmA, &full[stage], kb * C::BK,
                              (int)((t - 1) * p.mpad + (long)tm * C::BM));
              tc::tma_load_2d(sb(stage), &tmB, &full[stage], kb * C::BK,
                              (int)((u - 1) * p.npad + (long)tn * C::BN));
              ++issued;
              if (++stage == STAGES) { stage = 0; phase ^= 1; }
            }
          }
        }
      }
    }
    int pending = issued < STAGES ? issued : STAGES;
    for (int q = 0; q < pending; ++q) {
      if (--stage < 0) { stage = STAGES - 1; phase ^= 1; }
      if (!tc::mbar_wait_drain(&full[stage], phase)) break;
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t IDESC = tc::idesc_s8(C::HALF_ROWS, C::BN);
    int stage = 0;
    uint32_t phase = 0, acc_phase = 0;
    bool ok = true, any = false;
    for (int idx = blockIdx.x; idx < num_tiles && ok; idx += gridDim.x) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      for (int c0 = kb0; c0 < kb1 && ok; c0 += KCHUNK) {
        const int c1 = min(kb1, c0 + KCHUNK);
        for (int ph = 0; ph < S && ok; ++ph) {
          int t0, t1, d;
          oz_pairs<MOD>(S, ph, t0, t1, d);
          // The epilogue has drained the previous phase out of TMEM.
          if (!tc::mbar_wait(tempty, acc_phase ^ 1, abort_flag, p.err)) { ok = false; break; }
          tc::tc_fence_after();
          bool first = true;
          for (int t = t0; t <= t1 && ok; ++t) {
            for (int kb = c0; kb < c1; ++kb) {
              if (!tc::mbar_wait(&full[stage], phase, abort_flag, p.err)) { ok = false; break; }
              tc::tc_fence_after();
              const uint64_t a0 = tc::smem_desc(sa(stage), C::SWZ);
              const uint64_t a1 = tc::smem_desc(sa(stage) + C::HALF_ROWS * C::SWZ, C::SWZ);
              const uint64_t bd = tc::smem_desc(sb(stage), C::SWZ);
#pragma unroll
              for (int ks = 0; ks < C::KSTEPS; ++ks) {
                const uint64_t off = (uint64_t)((ks * 32) >> 4);
                tc::mma_i8(tmem_base, a0 + off, bd + off, IDESC, first ? 0u : 1u);
                tc::mma_i8(tmem_base + (uint32_t)C::BN, a1 + off, bd + off, IDESC, first ? 0u : 1u);
                first = false;
              }
              tc::mma_commit(&empty[stage]);
              any = true;
              if (++stage == STAGES) { stage = 0; phase ^= 1; }
            }
          }
          if (!ok) break;
          tc::mma_commit(tfull);
          acc_phase ^= 1;
        }
      }
    }
    if (any) {
      tc::mma_commit(drain);
      tc::mbar_wait(drain, 0, abort_flag, p.err);
    }
  }
  } else {
    tc::setmaxnreg_inc<TC_EPILOGUE_REGS>();
    // ---------------- epilogue ----------------
    // Warps 4-7 drain the accumulator of rows 0-127, warps 8-11 the one of
    // rows 128-255; each warp reads the TMEM lanes of its quadrant.
    const int quad = warp & 3, half = (warp - 4) >> 2;
    const int row = half * C::HALF_ROWS + quad * 32 + lane;  // tile row
    const uint32_t lane_base =
        tmem_base + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * C::BN);
    double *W = (double *)p.work + (size_t)blockIdx.x * C::BM * C::BN;
    // Residue workspace of the modular form: [l][16-column chunk][row][16 B],
    // so a warp's 16-byte stores and loads are 512 contiguous bytes.
    unsigned char *R = (unsigned char *)p.work + (size_t)blockIdx.x * S * C::BM * C::BN;
    uint32_t acc_phase = 0;
    bool ok = true;
    for (int idx = blockIdx.x; idx < num_tiles && ok; idx += gridDim.x) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      const long gi = (long)tm * C::BM + row;
      const bool row_ok = gi < w.m;
      const int ei = row_ok ? p.aexp[gi] : 0;
      if (kb0 >= kb1) {  // no update: beta * C
        if (row_ok)
          for (int j = 0; j < C::BN; ++j) {
            const long gj = (long)tn * C::BN + j;
            if (gj >= w.n || !b200_rel(w.ji, gj, gi)) continue;
            TC *cij = (TC *)p.c + gi * p.rs_c + gj * p.cs_c;
            *cij = p.beta != 0.0 ? (TC)(p.beta * (double)*cij) : TC(0);
          }
        continue;
      }
      const int nchunks = (kb1 - kb0 + KCHUNK - 1) / KCHUNK;
      const int nph = nchunks * S;
      int ph = 0;
      for (int cc = 0; cc < nchunks && ok; ++cc) {
        for (int pl = 0; pl < S; ++pl, ++ph) {
          int wok = tc::mbar_wait(tfull, acc_phase, abort_flag, p.err);
          if (!__all_sync(0xffffffffu, wok)) { ok = false; break; }
          tc::tc_fence_after();
          const bool last = ph == nph - 1;
          if constexpr (MOD) {
            const int m = p.crt.m[pl], bias = p.crt.bias[pl];
            const unsigned mg = p.crt.mg[pl];
            uint4 *Rl = (uint4 *)(R + (size_t)pl * C::BM * C::BN) + row;
            // Four 16-column TMEM loads in flight per wait: one round trip
            // per 64 columns instead of one per 16.
#pragma unroll
            for (int ch0 = 0; ch0 < C::BN / 16; ch0 += 4) {
              uint32_t rb[4][16];
#pragma unroll
              for (int q = 0; q < 4; ++q)
                tc::tmem_ld16(lane_base + (uint32_t)((ch0 + q) * 16), rb[q]);
              uint4 prev[4];
#pragma unroll
              for (int q = 0; q < 4; ++q)
                prev[q] = cc > 0 ? Rl[(ch0 + q) * C::BM] : make_uint4(0, 0, 0, 0);
              tc::tmem_wait_ld();
#pragma unroll
              for (int q = 0; q < 4; ++q) tc::tmem_tie16(rb[q]);
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                uint32_t out[4] = {0, 0, 0, 0};
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                  int res = b200_sym_mod((int)rb[q][j], m, mg, bias);  // |C'_l| <= 2^29
                  if (cc > 0) {
                    const uint4 pv = prev[q];
                    const uint32_t word = j < 4 ? pv.x : j < 8 ? pv.y : j < 12 ? pv.z : pv.w;
                    res = b200_sym_mod(res + (int)(int8_t)(word >> (8 * (j & 3))), m, mg, bias);
                  }
                  out[j >> 2] |= (uint32_t)(res & 0xff) << (8 * (j & 3));
                }
                Rl[(ch0 + q) * C::BM] = make_uint4(out[0], out[1], out[2], out[3]);
              }
            }
          } else {
#pragma unroll 1
            for (int ch = 0; ch < C::BN / 16; ++ch) {
              uint32_t r[16];
              tc::tmem_ld16(lane_base + (uint32_t)(ch * 16), r);
              tc::tmem_wait_ld();
              if (!row_ok) continue;
              // The chunk's loads (workspace, and in the last phase C and the
              // column scales) are issued before its stores.
              double wv[16], cv[16];
              int sc[16];
#pragma unroll
              for (int j = 0; j < 16; ++j) {
                const int col = ch * 16 + j;
                wv[j] = ph > 0 ? W[row + (size_t)col * C::BM] : 0.0;
                const long gj = (long)tn * C::BN + col;
                const bool in = last && gj < w.n && b200_rel(w.ji, gj, gi);
                cv[j] = in && p.beta != 0.0 ? (double)((const TC *)p.c)[gi * p.rs_c + gj * p.cs_c]
                                            : 0.0;
                sc[j] = in ? p.bexp[gj] : 0;
              }
#pragma unroll
              for (int j = 0; j < 16; ++j) {
                const int col = ch * 16 + j;
                double v = ldexp((double)(int)r[j], -7 * (S + 1 - pl));
                if (ph > 0) v += wv[j];
                if (!last) {
                  W[row + (size_t)col * C::BM] = v;
                  continue;
                }
                const long gj = (long)tn * C::BN + col;
                if (gj >= w.n || !b200_rel(w.ji, gj, gi)) continue;
                double out = p.alpha * b200_pow2_scale(v, ei + sc[j]);
                if (p.beta != 0.0) out = fma(p.beta, cv[j], out);
                ((TC *)p.c)[gi * p.rs_c + gj * p.cs_c] = (TC)out;
              }
            }
          }
          tc::tc_fence_before();
          tc::mbar_arrive(tempty);
          acc_phase ^= 1;
        }
      }
      if constexpr (MOD) {
        // TMEM is released; reconstruct C' from this thread's own residues
        // while the MMAs of the next tile run.
        if (!ok || !row_ok) continue;
        const OzCrt &k = p.crt;
        const int sh = ei - k.bits;
#pragma unroll 1
        for (int ch8 = 0; ch8 < C::BN / 8; ++ch8) {
          double s0[8], s1[8], s2[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) s0[j] = s1[j] = s2[j] = 0.0;
          const uint2 *base = (const uint2 *)((const uint4 *)R + (size_t)(ch8 >> 1) * C::BM + row) +
                              (ch8 & 1);
          // All residue loads of the chunk first (independent, one round
          // trip), then the arithmetic: a load-use chain per modulus would
          // serialise N L2/HBM latencies per chunk.
          uint2 rv[B200_MAX_MODULI];
#pragma unroll
          for (int l = 0; l < B200_MAX_MODULI; ++l)
            rv[l] = l < S ? base[(size_t)l * (C::BM * C::BN / 8)] : make_uint2(0, 0);
          // The chunk's C values and column scales load with the residues,
          // before any of its stores (one round trip, not one per element).
          TC cv[8];
          int sc[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const long gj = (long)tn * C::BN + ch8 * 8 + j;
            const bool in = gj < w.n && b200_rel(w.ji, gj, gi);
            cv[j] = in && p.beta != 0.0 ? ((const TC *)p.c)[gi * p.rs_c + gj * p.cs_c] : TC(0);
            sc[j] = in ? p.bexp[gj] : 0;
          }
#pragma unroll
          for (int l = 0; l < B200_MAX_MODULI; ++l) {
            if (l >= S) break;
            const uint2 v = rv[l];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const double rr = (double)(int8_t)((j < 4 ? v.x : v.y) >> (8 * (j & 3)));
              s0[j] = fma(rr, k.w[l][0], s0[j]);
              s1[j] = fma(rr, k.w[l][1], s1[j]);
              s2[j] = fma(rr, k.w[l][2], s2[j]);
            }
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const long gj = (long)tn * C::BN + ch8 * 8 + j;
            if (gj >= w.n || !b200_rel(w.ji, gj, gi)) continue;
            const double cp = oz_crt(k, s0[j], s1[j], s2[j]);
            double out = p.alpha * b200_pow2_scale(cp, sh + sc[j]);
            if (p.beta != 0.0) out = fma(p.beta, (double)cv[j], out);
            ((TC *)p.c)[gi * p.rs_c + gj * p.cs_c] = (TC)out;
          }
        }
      }
    }
  }

  tc::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem_base, C::TMEM_COLS);
  }
}

// ---- modular form on CTA pairs ------------------------------------------------
//
// tc_ozaki_kernel<true> with the 256 x 256 tile on a pair of SMs (cluster
// of two, cta_group::2): each CTA loads its 128 rows of op(A) and 128 rows
// (tile columns) of op(B) into its own shared memory, the leader issues one
// M = 256, N = 256 int8 MMA per k-step, and each CTA's TMEM holds its 128
// accumulator rows x 256 columns -- half of what one CTA of the single-SM
// kernel needs, so two accumulators fit and the epilogue's reduction of
// modulus l overlaps the MMAs of modulus l + 1 (the single-SM kernel's
// issuer waits for every drain).  Residues, CRT and the output are the
// single-SM kernel's, element by element.
struct OzPairCfg {
  static constexpr int BM = 128, BN = 128, SWZ = 128, BK = 128, STAGES = 6;  // per CTA
  static constexpr int TILE_M = 256, TILE_N = 256;
  static constexpr int A_TILE = BM * SWZ, B_TILE = BN * SWZ;
  static constexpr int STAGE_BYTES = A_TILE + B_TILE;
  static constexpr int KSTEPS = SWZ / 32;
  static constexpr int THREADS = 384, EPI_WARPS = 8;
  static constexpr int HALF = TILE_N / 2;  // columns per epilogue thread
  static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 + 256;
  static constexpr uint32_t TMEM_COLS = 512;
};

template <typename TC>
__global__ void __launch_bounds__(384, 1)
    tc_ozaki2_pair_kernel(const __grid_constant__ CUtensorMap tmA,
                          const __grid_constant__ CUtensorMap tmB, const __grid_constant__ OzParams p) {
  using C = OzPairCfg;
  constexpr int STAGES = C::STAGES;
  constexpr int KCHUNK = OZ2_KCHUNK / C::BK;  // in k-blocks
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char *smem =
      (unsigned char *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(smem + STAGES * C::STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *tfull = empty + STAGES;
  uint64_t *tempty = tfull + 2;
  uint64_t *drain = tempty + 2;
  uint32_t *tmem_slot = (uint32_t *)(drain + 1);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = tc::cluster_rank();
  const bool leader = rank == 0;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      tc::mbar_init(&tfull[a], 1);
      tc::mbar_init(&tempty[a], 2 * C::EPI_WARPS);
    }
    tc::mbar_init(drain, 1);
    *abort_flag = 0;
    tc::fence_barrier_init();
    tc::tma_prefetch_desc(&tmA);
    tc::tma_prefetch_desc(&tmB);
  }
  if (warp == 2) tc::tmem_alloc_pair(tmem_slot, C::TMEM_COLS);
  tc::tc_fence_before();
  __syncthreads();
  tc::cluster_sync();
  tc::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  const TileWalk &w = p.w;  // bm = bn = 256: pair tiles
  const int S = p.slices;   // modulus count
  const int num_tiles = w.tiles_m * w.tiles_n;
  const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
  auto sa = [&](int st) { return smem + st * C::STAGE_BYTES; };
  auto sb = [&](int st) { return smem + st * C::STAGE_BYTES + C::A_TILE; };

  if (warp < 4) {
  tc::setmaxnreg_dec<TC_PRODUCER_REGS>();
  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer (both CTAs) ----------------
    int stage = 0, issued = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (int idx = pair; idx < num_tiles && ok; idx += npairs) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      const long arow = (long)tm * C::TILE_M + rank * C::BM;
      const long brow = (long)tn * C::TILE_N + rank * C::BN;
      for (int c0 = kb0; c0 < kb1 && ok; c0 += KCHUNK) {
        const int c1 = min(kb1, c0 + KCHUNK);
        for (int l = 0; l < S && ok; ++l) {
          for (int kb = c0; kb < c1; ++kb) {
            if (!tc::mbar_wait(&empty[stage], phase ^ 1, abort_flag, p.err)) { ok = false; break; }
            if (leader) tc::mbar_arrive_expect_tx(&full[stage], 2 * C::STAGE_BYTES);
            const uint32_t fb = tc::map_rank(&full[stage], 0);
            tc::tma_load_2d_pair(sa(stage), &tmA, fb, kb * C::BK, (int)(l * p.mpad + arow));
            tc::tma_load_2d_pair(sb(stage), &tmB, fb, kb * C::BK, (int)(l * p.npad + brow));
            ++issued;
            if (++stage == STAGES) { stage = 0; phase ^= 1; }
          }
        }
      }
    }
    if (leader) {  // both CTAs' last loads complete on the leader's barriers
      int pending = issued < STAGES ? issued : STAGES;
      for (int q = 0; q < pending; ++q) {
        if (--stage < 0) { stage = STAGES - 1; phase ^= 1; }
        if (!tc::mbar_wait_drain(&full[stage], phase)) break;
      }
    }
  } else if (warp == 1 && lane == 0 && leader) {
    // ---------------- MMA issuer (leader) ----------------
    constexpr uint32_t IDESC = tc::idesc_s8(C::TILE_M, C::TILE_N);
    int stage = 0, acc = 0;
    uint32_t phase = 0, acc_phase = 0;
    bool ok = true, any = false;
    for (int idx = pair; idx < num_tiles && ok; idx += npairs) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      for (int c0 = kb0; c0 < kb1 && ok; c0 += KCHUNK) {
        const int c1 = min(kb1, c0 + KCHUNK);
        for (int l = 0; l < S && ok; ++l) {
          // Both CTAs' epilogues have reduced this accumulator's last use.
          if (!tc::mbar_wait(&tempty[acc], acc_phase ^ 1, abort_flag, p.err)) { ok = false; break; }
          tc::tc_fence_after();
          const uint32_t d = tmem_base + (uint32_t)(acc * C::TILE_N);
          bool first = true;
          for (int kb = c0; kb < c1; ++kb) {
            if (!tc::mbar_wait(&full[stage], phase, abort_flag, p.err)) { ok = false; break; }
            tc::tc_fence_after();
            const uint64_t ad = tc::smem_desc(sa(stage), C::SWZ);
            const uint64_t bd = tc::smem_desc(sb(stage), C::SWZ);
#pragma unroll
            for (int ks = 0; ks < C::KSTEPS; ++ks) {
              const uint64_t off = (uint64_t)((ks * 32) >> 4);
              tc::mma_i8_pair(d, ad + off, bd + off, IDESC, first ? 0u : 1u);
              first = false;
            }
            tc::mma_commit_pair(&empty[stage]);
            any = true;
            if (++stage == STAGES) { stage = 0; phase ^= 1; }
          }
          if (!ok) break;
          tc::mma_commit_pair(&tfull[acc]);
          if (++acc == 2) { acc = 0; acc_phase ^= 1; }
        }
      }
    }
    if (any) {
      tc::mma_commit_pair(drain);
      tc::mbar_wait(drain, 0, abort_flag, p.err);
    }
  }
  } else {
    tc::setmaxnreg_inc<TC_EPILOGUE_REGS>();
    // ---------------- epilogue (both CTAs: this CTA's 128 rows) ----------------
    // Warps 4-7 take columns 0-127 of the tile, warps 8-11 columns 128-255;
    // each warp reads the TMEM lanes of its quadrant.
    const int quad = warp & 3, hc = (warp - 4) >> 2;
    const int row = quad * 32 + lane;  // row within this CTA's half of the tile
    const uint32_t lane_base = tmem_base + ((uint32_t)(quad * 32) << 16) + (uint32_t)(hc * C::HALF);
    // Residue workspace: [l][16-column chunk][row][16 B] for this CTA's 128
    // rows, so a warp's 16-byte stores and loads are 512 contiguous bytes.
    unsigned char *R = (unsigned char *)p.work + (size_t)blockIdx.x * S * C::BM * C::TILE_N;
    int acc = 0;
    uint32_t acc_phase = 0;
    bool ok = true;
    for (int idx = pair; idx < num_tiles && ok; idx += npairs) {
      int tm, tn, kb0, kb1;
      w.coords(idx, tm, tn);
      if (!w.valid(tm, tn)) continue;
      w.krange(tm, tn, kb0, kb1);
      const long gi = (long)tm * C::TILE_M + rank * C::BM + row;
      const bool row_ok = gi < w.m;
      const int ei = row_ok ? p.aexp[gi] : 0;
      const long gj0 = (long)tn * C::TILE_N + hc * C::HALF;
      if (kb0 >= kb1) {  // no update: beta * C
        if (row_ok)
          for (int j = 0; j < C::HALF; ++j) {
            const long gj = gj0 + j;
            if (gj >= w.n || !b200_rel(w.ji, gj, gi)) continue;
            TC *cij = (TC *)p.c + gi * p.rs_c + gj * p.cs_c;
            *cij = p.beta != 0.0 ? (TC)(p.beta * (double)*cij) : TC(0);
          }
        continue;
      }
      const int nchunks = (kb1 - kb0 + KCHUNK - 1) / KCHUNK;
      for (int cc = 0; cc < nchunks && ok; ++cc) {
        for (int l = 0; l < S; ++l) {
          int wok = tc::mbar_wait(&tfull[acc], acc_phase, abort_flag, p.err);
          if (!__all_sync(0xffffffffu, wok)) { ok = false; break; }
          tc::tc_fence_after();
          const int m = p.crt.m[l], bias = p.crt.bias[l];
          const unsigned mg = p.crt.mg[l];
          uint4 *Rl = (uint4 *)(R + (size_t)l * C::BM * C::TILE_N) + row;
          const uint32_t base = lane_base + (uint32_t)(acc * C::TILE_N);
#pragma unroll
          for (int ch0 = 0; ch0 < C::HALF / 16; ch0 += 4) {
            uint32_t rb[4][16];
#pragma unroll
            for (int q = 0; q < 4; ++q) tc::tmem_ld16(base + (uint32_t)((ch0 + q) * 16), rb[q]);
            const int chunk0 = hc * (C::HALF / 16) + ch0;  // 16-column chunk of the tile
            uint4 prev[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
              prev[q] = cc > 0 ? Rl[(chunk0 + q) * C::BM] : make_uint4(0, 0, 0, 0);
            tc::tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 4; ++q) tc::tmem_tie16(rb[q]);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              uint32_t out[4] = {0, 0, 0, 0};
#pragma unroll
              for (int j = 0; j < 16; ++j) {
                int res = b200_sym_mod((int)rb[q][j], m, mg, bias);  // |C'_l| <= 2^29
                if (cc > 0) {
                  const uint4 pv = prev[q];
                  const uint32_t word = j < 4 ? pv.x : j < 8 ? pv.y : j < 12 ? pv.z : pv.w;
                  res = b200_sym_mod(res + (int)(int8_t)(word >> (8 * (j & 3))), m, mg, bias);
                }
                out[j >> 2] |= (uint32_t)(res & 0xff) << (8 * (j & 3));
              }
              Rl[(chunk0 + q) * C::BM] = make_uint4(out[0], out[1], out[2], out[3]);
            }
          }
          tc::tc_fence_before();
          __syncwarp();
          if (lane == 0) tc::mbar_arrive_cluster(tc::map_rank(&tempty[acc], 0));
          if (++acc == 2) { acc = 0; acc_phase ^= 1; }
        }
      }
      // The tile's accumulators are released; reconstruct C' from this
      // thread's own residues while the MMAs of the next tile run.
      if (!ok || !row_ok) continue;
      const OzCrt &k = p.crt;
      const int sh = ei - k.bits;
#pragma unroll 1
      for (int ch8 = 0; ch8 < C::HALF / 8; ++ch8) {
        double s0[8], s1[8], s2[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) s0[j] = s1[j] = s2[j] = 0.0;
        const int col8 = hc * (C::HALF / 8) + ch8;  // 8-column group of the tile
        const uint2 *rbase =
            (const uint2 *)((const uint4 *)R + (size_t)(col8 >> 1) * C::BM + row) + (col8 & 1);
        uint2 rv[B200_MAX_MODULI];
#pragma unroll
        for (int l = 0; l < B200_MAX_MODULI; ++l)
          rv[l] = l < S ? rbase[(size_t)l * (C::BM * C::TILE_N / 8)] : make_uint2(0, 0);
        TC cv[8];
        int sc[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const long gj = gj0 + ch8 * 8 + j;
          const bool in = gj < w.n && b200_rel(w.ji, gj, gi);
          cv[j] = in && p.beta != 0.0 ? ((const TC *)p.c)[gi * p.rs_c + gj * p.cs_c] : TC(0);
          sc[j] = in ? p.bexp[gj] : 0;
        }
#pragma unroll
        for (int l = 0; l < B200_MAX_MODULI; ++l) {
          if (l >= S) break;
          const uint2 v = rv[l];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const double rr = (double)(int8_t)((j < 4 ? v.x : v.y) >> (8 * (j & 3)));
            s0[j] = fma(rr, k.w[l][0], s0[j]);
            s1[j] = fma(rr, k.w[l][1], s1[j]);
            s2[j] = fma(rr, k.w[l][2], s2[j]);
          }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const long gj = gj0 + ch8 * 8 + j;
          if (gj >= w.n || !b200_rel(w.ji, gj, gi)) continue;
          const double cp = oz_crt(k, s0[j], s1[j], s2[j]);
          double out = p.alpha * b200_pow2_scale(cp, sh + sc[j]);
          if (p.beta != 0.0) out = fma(p.beta, (double)cv[j], out);
          ((TC *)p.c)[gi * p.rs_c + gj * p.cs_c] = (TC)out;
        }
      }
    }
  }

  tc::tc_fence_before();
  __syncthreads();
  tc::cluster_sync();
  if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc_pair(tmem_base, C::TMEM_COLS);
  }
}

// The modular form's moduli: the largest pairwise coprime integers <= 256.
constexpr int OZ2_MODULI[B200_MAX_MODULI] = {256, 255, 253, 251, 247, 241, 239, 233,
                                             229, 227, 223, 217, 211, 199, 197, 193};

// Host set-up of the modular form for N moduli and inner dimension k: the
// residue constants for packing and the epilogue, the CRT levels, and the
// scale exponents pa (rows of op(A)) and pb (columns of op(B)), each at most
// pmax (bits beyond the input's significand buy nothing).
int oz2_setup(int N, long k, int pmax, B200Moduli *mod, OzCrt *crt, int *pa, int *pb) {
  typedef unsigned __int128 u128;
  u128 M = 1;
  for (int l = 0; l < N; ++l) M *= (u128)OZ2_MODULI[l];
  long double log2m = 0.0L;
  for (int l = 0; l < N; ++l) log2m += log2l((long double)OZ2_MODULI[l]);
  // k 2^(pa+pb) <= (M/2)(1 - 2^-30): the CRT rounding of q stays exact.
  const long double room = log2m - 1.0L - log2l((long double)(k > 0 ? k : 1)) - 1e-6L;
  const int total = (int)floorl(room);
  if (total < 16) return b200_set_error(B200_EINVAL, "ozaki2: too few moduli for this k");
  *pa = std::min(pmax, (total + 1) / 2);
  *pb = std::min(pmax, total - *pa);
  mod->n = N;
  memset(crt, 0, sizeof *crt);
  crt->bits = *pa + *pb;
  const u128 mask42 = (((u128)1) << 42) - 1;
  auto level = [&](u128 x, int lev) -> double {
    const int shift = 84 - 42 * lev;
    return ldexp((double)(unsigned long long)((x >> shift) & mask42), shift);
  };
  for (int l = 0; l < N; ++l) {
    const int m = OZ2_MODULI[l];
    mod->m[l] = crt->m[l] = m;
    mod->c19[l] = (int)((1u << 19) % (unsigned)m);
    mod->c38[l] = (int)((((u128)1) << 38) % (u128)m);
    mod->mg[l] = crt->mg[l] = (unsigned)(((1ull << 39) + (unsigned long long)m - 1) / m);
    mod->bias[l] = crt->bias[l] = m / 2 + (int)(((1u << 29) + m - 1) / m) * m;
    const u128 Ml = M / (u128)m;
    const int r = (int)(Ml % (u128)m);
    int y = 1;
    while ((r * y) % m != 1) ++y;  // m <= 256: a direct search is enough
    const u128 W = Ml * (u128)y;  // < M
    for (int lev = 0; lev < 3; ++lev) crt->w[l][lev] = level(W, lev);
  }
  for (int lev = 0; lev < 3; ++lev) crt->mlev[lev] = level(M, lev);
  crt->inv_m = (double)(1.0L / (long double)M);
  return B200_OK;
}

}  // namespace

namespace {

template <typename T>
cudaLaunchConfig_t oz2_pair_config(cudaLaunchAttribute *attr, int grid, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(OzPairCfg::THREADS);
  cfg.dynamicSmemBytes = OzPairCfg::SMEM;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

// Configures the pair kernel once (shared memory, register-split check) and
// returns how many CTA pairs can be resident at once.
template <typename T>
int oz2_pair_clusters(int *clusters) {
  static std::once_flag once;
  static int conf = B200_OK, cached = 0;
  B200_TRY(b200_once(once, conf, "ozaki2 pair kernel: set-up failed", []() -> int {
    auto kern = tc_ozaki2_pair_kernel<T>;
    B200_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       OzPairCfg::SMEM));
    cudaFuncAttributes fa;
    B200_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    if (OzPairCfg::THREADS != 384 || !tc_register_split_fits(fa.numRegs))
      return b200_set_error(B200_EINVAL, "ozaki2 pair kernel: register split does not fit its launch");
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = oz2_pair_config<T>(attr, 2 * b200_sm_count(), nullptr);
    if (cudaOccupancyMaxActiveClusters(&cached, (void *)kern, &cfg) != cudaSuccess || cached < 1) {
      cudaGetLastError();
      return b200_set_error(B200_ECUDA, "ozaki2 pair kernel: no CTA pair can be resident");
    }
    return B200_OK;
  }));
  *clusters = cached;
  return B200_OK;
}

template <typename T>
int launch_oz2_pair(const CUtensorMap &ta, const CUtensorMap &tb, const OzParams &p, int grid,
                    cudaStream_t s) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = oz2_pair_config<T>(attr, grid, s);
  B200ProfScope prof(sizeof(T) == 8 ? "tc_ozaki2_i8" : "tc_ozaki2_s_i8", s);
  B200_CUDA_TRY(cudaLaunchKernelEx(&cfg, tc_ozaki2_pair_kernel<T>, ta, tb, p));
  return B200_OK;
}

template <typename T>
int run_ozaki(const b200_l3_desc_t *d, bool mod) {
  using C = OzCfg;
  constexpr bool F64 = sizeof(T) == 8;
  int slices = d->slices > 0 ? d->slices : b200_get_default_slices(d->dtype);
  if (slices <= 0) slices = mod ? (F64 ? B200_MAX_MODULI : 8) : 7;
  if (!mod && (slices < 2 || slices > OZ_MAX_SLICES))
    return b200_set_error(B200_EINVAL, "ozaki: slice count must be in [2, 12]");
  if (mod && (slices < 6 || slices > B200_MAX_MODULI))
    return b200_set_error(B200_EINVAL, "ozaki2: modulus count must be in [6, 16]");
  cudaStream_t s = b200_cur_stream();
  const long ktot = (long)d->k * d->npairs;
  const long mpad = b200_round_up(d->m, C::BM), npad = b200_round_up(d->n, C::BN);
  const long kpad = b200_round_up(ktot, C::BK);
  if (slices * (mpad > npad ? mpad : npad) > 0x7fffffffL)
    return b200_set_error(B200_EINVAL, "ozaki form: operand too large for 32-bit TMA rows");
  OzParams p;
  memset(&p, 0, sizeof p);
  B200Moduli moduli;
  memset(&moduli, 0, sizeof moduli);
  int pa = 0, pb = 0;
  // FP64 inputs carry 53 significant bits, FP32 inputs 24: a few bits more
  // than that keeps elements a few binades below the row maximum exact.
  if (mod) B200_TRY(oz2_setup(slices, ktot, F64 ? 56 : 27, &moduli, &p.crt, &pa, &pb));
  const int sms = b200_sm_count();
  const int tiles = (int)((mpad / C::BM) * (npad / C::BN));
  // The modular form runs on CTA pairs (tc_ozaki2_pair_kernel) below 576
  // tiles (24^2: up to ~6000^2 outputs), unless MUBLIS_B200_TC_PAIR=0; grid
  // then counts CTAs, two per tile slot.  Measured kernel times, pair vs
  // one SM per tile: 2048^3 0.18 vs 0.38 ms (the 64 tiles keep 128 SMs busy
  // instead of 64), 3072^3 0.43 vs 0.48, 4096^3 1.02 vs 1.09, 6144^3 2.90
  // vs 2.91, 8192^3 6.70 vs 6.45.  Results are bit-identical either way.
  static const bool pair_on = [] {
    const char *e = getenv("MUBLIS_B200_TC_PAIR");
    return !(e && !strcmp(e, "0"));
  }();
  const bool pair = mod && pair_on && tiles < 576;
  int grid = tiles < sms ? tiles : sms;
  if (pair) {
    int clusters = 0;
    B200_TRY(oz2_pair_clusters<T>(&clusters));
    grid = 2 * (tiles < clusters ? tiles : clusters);
  }

  void *ap = nullptr, *bp = nullptr, *amax = nullptr, *bmax = nullptr, *work = nullptr;
  int st = b200_alloc(&amax, (sizeof(unsigned long long) + sizeof(int)) * (mpad + npad));
  int *exps = nullptr;
  if (st == B200_OK) {
    bmax = (unsigned long long *)amax + mpad;
    exps = (int *)((unsigned long long *)amax + mpad + npad);
    st = cudaMemsetAsync(amax, 0, sizeof(unsigned long long) * (mpad + npad), s) == cudaSuccess
             ? B200_OK
             : b200_set_error(B200_ECUDA, "memset failed");
  }
  if (st == B200_OK) st = b200_alloc(&ap, (size_t)slices * mpad * kpad);
  if (st == B200_OK) st = b200_alloc(&bp, (size_t)slices * npad * kpad);
  const size_t work_bytes = pair ? (size_t)grid * slices * OzPairCfg::BM * OzPairCfg::TILE_N
                            : mod  ? (size_t)grid * slices * C::BM * C::BN
                                   : sizeof(double) * grid * C::BM * C::BN;
  if (st == B200_OK) st = b200_alloc(&work, work_bytes);
  const mublis_l3_product_t &pr = d->product;
  PackView va[2], vb[2];
  for (int t = 0; t < d->npairs; ++t) {
    va[t] = PackView{d->a[t], d->rs_a[t], d->cs_a[t], (int)pr.a.struc, (int)pr.a.uplo,
                     (int)pr.a.diag, (int)pr.domain.pi};
    vb[t] = PackView{d->b[t], d->rs_b[t], d->cs_b[t], (int)pr.b.struc, (int)pr.b.uplo,
                     (int)pr.b.diag, (int)pr.domain.jp};
  }
  // Scales over the whole (concatenated) k of every row / column.
  for (int t = 0; t < d->npairs && st == B200_OK; ++t) {
    st = launch_absmax<T>(va[t], false, d->m, d->k, (unsigned long long *)amax, s);
    if (st == B200_OK)
      st = launch_absmax<T>(vb[t], true, d->n, d->k, (unsigned long long *)bmax, s);
  }
  if (st == B200_OK) st = launch_scale_exps((const unsigned long long *)amax, exps, mpad + npad, s);
  for (int t = 0; t < d->npairs && st == B200_OK; ++t) {
    long kk0 = (long)t * d->k, kk1 = t + 1 == d->npairs ? kpad : kk0 + d->k;
    const int xform = mod ? PACK_INT8_MODULI : PACK_INT8_SLICES;
    PackOut oa{ap, kpad, mpad * kpad, PACK_K_MAJOR, xform, slices,
               (const unsigned long long *)amax, pa, moduli};
    PackOut ob{bp, kpad, npad * kpad, PACK_K_MAJOR, xform, slices,
               (const unsigned long long *)bmax, pb, moduli};
    st = launch_pack<T>(va[t], false, d->m, d->k, mpad, kk0, kk1, oa, s);
    if (st == B200_OK) st = launch_pack<T>(vb[t], true, d->n, d->k, npad, kk0, kk1, ob, s);
  }
  CUtensorMap ta, tb;
  // Boxes of one CTA's share of a tile: 256 rows, or 128 on CTA pairs.
  const int box = pair ? OzPairCfg::BM : C::BM;
  if (st == B200_OK) st = b200_make_tmap(&ta, ap, 0, kpad, slices * mpad, C::BK, box, C::SWZ);
  if (st == B200_OK) st = b200_make_tmap(&tb, bp, 0, kpad, slices * npad, C::BK, box, C::SWZ);
  if (st == B200_OK) {
    p.w.tiles_m = (int)(mpad / C::BM);
    p.w.tiles_n = (int)(npad / C::BN);
    p.w.bm = C::BM;
    p.w.bn = C::BN;
    p.w.m = d->m;
    p.w.n = d->n;
    p.w.k = ktot;
    p.w.bk = C::BK;
    p.w.kblocks = (int)(kpad / C::BK);
    p.w.jp = pr.domain.jp;
    p.w.ji = pr.domain.ji;
    p.w.pi = pr.domain.pi;
    p.mpad = mpad;
    p.npad = npad;
    p.slices = slices;
    p.alpha = d->alpha;
    p.beta = d->beta;
    p.c = d->c;
    p.rs_c = d->rs_c;
    p.cs_c = d->cs_c;
    p.work = work;
    p.aexp = exps;
    p.bexp = exps + mpad;
    p.err = b200_device_error_word();
    if (pair) {
      st = launch_oz2_pair<T>(ta, tb, p, grid, s);
      b200_free(ap);
      b200_free(bp);
      b200_free(work);
      b200_free(amax);
      return st;
    }
    auto kern = tc_ozaki_kernel<true, T>;
    if constexpr (F64) {
      if (!mod) kern = tc_ozaki_kernel<false, double>;
    }
    static std::once_flag once[2];
    static int conf[2] = {B200_OK, B200_OK};
    if (st == B200_OK)
      st = b200_once(once[mod], conf[mod], "ozaki kernel: set-up failed", [&]() -> int {
        B200_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           C::SMEM));
        // The warpgroup register split must fit the compiled allocation (an
        // increase that cannot be granted would wait forever).
        cudaFuncAttributes fa;
        B200_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
        if (C::THREADS != 384 || !tc_register_split_fits(fa.numRegs))
          return b200_set_error(B200_EINVAL, "ozaki kernel: register split does not fit its launch");
        return B200_OK;
      });
    if (st == B200_OK) {
      B200ProfScope prof(mod ? (F64 ? "tc_ozaki2_i8" : "tc_ozaki2_s_i8") : "tc_ozaki_i8", s);
      kern<<<grid, C::THREADS, C::SMEM, s>>>(ta, tb, p);
      if (cudaGetLastError() != cudaSuccess) st = b200_set_error(B200_ECUDA, "ozaki launch failed");
    }
  }
  b200_free(ap);
  b200_free(bp);
  b200_free(work);
  b200_free(amax);
  return st;
}

}  // namespace

int tc_run_ozaki(const b200_l3_desc_t *d) {
  const bool mod = d->form == B200_FORM_OZAKI2;
  if (d->dtype == B200_F64) return run_ozaki<double>(d, mod);
  if (!mod) return b200_set_error(B200_EINVAL, "the slice Ozaki form is FP64-only");
  return run_ozaki<float>(d, true);
}
