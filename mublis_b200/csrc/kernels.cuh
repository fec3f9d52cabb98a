// kernels.cuh -- launchers shared between the CUDA translation units.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <vector>

#include "common.cuh"

// Logical operand view for packing.  Element (r, c) of the stored operand
// lives at x[r * rs + c * cs]; `struc/uplo/diag` give its logical view
// (frame/l1m/packm.c:40-71) and `mask_rel` a domain relation applied as
// rel(mask_rel, c, r) (pi on A's (i, p) or jp on B's (p, j)).
struct PackView {
  const void *x;
  long rs, cs;
  int struc, uplo, diag;
  int mask_rel;
};

// Logical element (r, c) of a view (frame/l1m/packm.c:40-71): zero outside
// the mask relation, the stored triangle reflected for a symmetric operand,
// zero outside it for a triangular one (unit / inverted diagonal applied).
// Elements outside the stored triangle are never read.
template <typename T>
__device__ __forceinline__ T load_logical(const PackView &v, long r, long c) {
  const T *x = (const T *)v.x;
  if (!b200_rel(v.mask_rel, c, r)) return T(0);
  long delta = r - c;
  bool stored = v.uplo == MUBLIS_LOWER ? delta >= 0 : (v.uplo == MUBLIS_UPPER ? delta <= 0 : true);
  if (v.struc == MUBLIS_STRUC_SYMMETRIC) {
    return stored ? x[r * v.rs + c * v.cs] : x[c * v.rs + r * v.cs];
  }
  if (v.struc == MUBLIS_STRUC_TRIANGULAR) {
    if (!stored) return T(0);
    if (delta == 0 && v.diag == MUBLIS_PACKM_DIAG_UNIT) return T(1);
    T val = x[r * v.rs + c * v.cs];
    if (delta == 0 && v.diag == MUBLIS_PACKM_DIAG_INVERT) val = T(1) / val;
    return val;
  }
  return x[r * v.rs + c * v.cs];
}

// Output orientation of a packed panel.  The panel covers mn in [0, mn_pad)
// and kk in [kk0, kk1); logical element (mn, kk - kk0) is taken from the
// view, as (r, c) = (mn, kk) for an A-side view or (kk, mn) for a B-side
// view; anything past mn_len / k_len is zero.
enum PackLayout {
  PACK_MN_MAJOR = 0,  // out[kk * ld + mn]       (SIMT kernels)
  PACK_K_MAJOR = 1,   // out[mn * ld + kk]       (tcgen05 kernels)
  PACK_FRAG64 = 2     // doubles in mma.m16n8k4 fragment order (FP64 MMA
                      // kernel), ld = Kpad: see b200_frag64_offset
};

// Offset of element (mn, kk) of a PACK_FRAG64 panel (Kpad = ld, a multiple
// of 16; Mpad a multiple of 128).  The panel is a sequence of 128-row
// strips; a strip is a sequence of k-quads (4 consecutive kk); a k-quad of a
// strip is 8 blocks of 16 rows, each 32 lanes x 2 doubles in the order an
// mma.m16n8k4 .f64 fragment is held: lane = 4 (mn % 8) + kk % 4 holds rows
// mn % 16 < 8 and >= 8 of its block as one 16-byte pair.  An A operand
// strip is a 16-row block fragment (a0, a1) per lane; a B operand strip is
// two 8-column fragments (b0 of columns 0-7, b0 of columns 8-15) per lane.
// So one k-block of 16 of one strip is 16 KB contiguous, and every warp
// fragment load is 512 contiguous bytes.
__host__ __device__ inline long b200_frag64_offset(long mn, long kk, long kpad) {
  return (((((mn >> 7) * (kpad >> 2) + (kk >> 2)) * 8 + ((mn & 127) >> 4)) * 32 +
           (((mn & 7) << 2) | (kk & 3))) << 1) |
         ((mn >> 3) & 1);
}

enum PackXform {
  PACK_COPY = 0,         // T -> T
  PACK_BF16_SPLIT = 1,   // f32 -> `terms` bf16 planes (hi, lo[, lo2])
  PACK_INT8_SLICES = 2,  // f64 -> `terms` int8 planes of 7-bit slices of
                         // x * 2^(7 - e), e from the row/column abs-max
  PACK_INT8_MODULI = 3,  // f64 -> `terms` int8 planes: the symmetric residues
                         // of X = rint(x * 2^(bits - e)) modulo each modulus
  PACK_FP16_SPLIT = 4    // f32 -> 2 fp16 planes of xs = x * 2^(15 - e) (e from
                         // the row/column abs-max, |xs| < 2^15): hi = rn(xs),
                         // lo = rn(xs - hi)
};

// fp16 split scaling: the row/column maximum lands just below 2^15, so that
// lo = rn(xs - hi) (about 2^-11 |xs|) stays a normal fp16 number for every
// element down to 2^-18 of its row's maximum (fp16 normals start at 2^-14;
// the tensor cores ran the product noticeably slower on subnormal halves).
constexpr int B200_FP16_SCALE_EXP = 15;

// Pairwise coprime moduli (<= 256) of the modular (CRT) Ozaki form and the
// constants that reduce an integer modulo each of them without division:
// c19/c38 = 2^19/2^38 mod m; mg = ceil(2^39 / m); bias = floor(m/2) + K m
// with K m >= 2^29 (see b200_sym_mod).
constexpr int B200_MAX_MODULI = 16;
struct B200Moduli {
  int n;
  int m[B200_MAX_MODULI], c19[B200_MAX_MODULI], c38[B200_MAX_MODULI], bias[B200_MAX_MODULI];
  unsigned mg[B200_MAX_MODULI];
};

struct PackOut {
  void *out;
  long ld;
  long plane_stride;  // elements between planes
  int layout, xform, terms;
  const unsigned long long *absmax;  // INT8 forms: bits of max |x| per mn
  int bits;                          // PACK_INT8_MODULI: |X| <= 2^bits
  B200Moduli mod;                    // PACK_INT8_MODULI
};

// Symmetric residue of t modulo m, in [-floor(m/2), m - 1 - floor(m/2)]
// (within [-128, 127] for m <= 256), for |t| <= 2^29.  u = t + bias lies in
// [0, 2^31); for u < 2^31 and m <= 2^8, floor(u / m) = umulhi(u, mg) >> 7
// with mg = ceil(2^39 / m) exactly (Granlund and Montgomery 1994: the error
// u (mg m - 2^39) / (m 2^39) stays below 1/m; for m = 256 mg is exact), so
// r = u - q m - floor(m/2) needs no correction.
__device__ __forceinline__ int b200_sym_mod(int t, int m, unsigned mg, int bias) {
  const unsigned u = (unsigned)(t + bias);
  const unsigned q = __umulhi(u, mg) >> 7;
  return (int)(u - q * (unsigned)m) - (m >> 1);
}

template <typename T>
int launch_absmax(const PackView &v, bool b_side, long mn_len, long k_len,
                  unsigned long long *absmax, cudaStream_t s);

// exps[i] = b200_scale_exp(absmax[i]) for i < count: the epilogues read one
// int per row / column instead of a 64-bit abs-max and its frexp.
int launch_scale_exps(const unsigned long long *absmax, int *exps, long count, cudaStream_t s);

// Exponent e with max|x| < 2^e (frexp), 0 for an all-zero row.
__device__ inline int b200_scale_exp(unsigned long long absmax_bits) {
  if (absmax_bits == 0) return 0;
  int e;
  frexp(__longlong_as_double((long long)absmax_bits), &e);
  return e;
}

// x * 2^e rounded once.
//  * float: the product is formed exactly in FP64 and rounded once to float;
//    valid for -1022 <= e <= 1023 (the fp16x3 epilogue's e = e_i + f_j - 30
//    stays within [-330, 230] for FP32 inputs).
//  * double: one multiply by the exact power of two where 2^e is a normal
//    number, else ldexp.
__device__ __forceinline__ float b200_pow2_scale(float x, int e) {
  return (float)((double)x * __longlong_as_double((long long)(e + 1023) << 52));
}
__device__ __forceinline__ double b200_pow2_scale(double x, int e) {
  return e >= -1022 && e <= 1023 ? x * __longlong_as_double((long long)(e + 1023) << 52)
                                 : ldexp(x, e);
}

template <typename T>
int launch_pack(const PackView &v, bool b_side, long mn_len, long k_len, long mn_pad,
                long kk0, long kk1, const PackOut &o, cudaStream_t s);

// Plain FP32 / FP64 GEMM on the FMA pipes over packed MN-major panels.
template <typename T>
struct SimtGemmArgs {
  const T *ap;  // [Kpad][Mpad]
  const T *bp;  // [Kpad][Npad]
  long lda, ldb;
  T *c;
  long rs_c, cs_c;
  int m, n, k;
  T alpha, beta;
  int jp, ji, pi;
  // Scheduling, filled by the launcher when the caller passes a SimtPolicy:
  // persistent CTAs take units (tile, k-chunk) from a counter.  Left at
  // these defaults, every CTA computes the one tile of its block index.
  const int2 *tile_list = nullptr;  // (tm, tn) of the tiles to compute, or null: all tiles
  int ntiles = 0;                   // tiles scheduled (0: all tiles, one per CTA)
  int splits = 1;                   // k-chunks per tile (split-K)
  int *work = nullptr;              // unit counter (zeroed): persistent CTAs
  int *arrivals = nullptr;          // per tile: k-chunks finished (zeroed), splits > 1
  T *partials = nullptr;            // per unit: its k-chunk's sums, splits > 1
};

// What the launcher needs to schedule a call on persistent CTAs with
// split-K: the whole call's output size (a column panel of a larger call
// carries the call's m and n, so every panel splits its tiles' k ranges as
// the whole call would, and panels stay bit-identical to the one-call
// result).
struct SimtPolicy {
  long m_full, n_full;
};

// Plain FP64 GEMM on the FP64 tensor pipe over PACK_FRAG64 panels.
struct DmmaGemmArgs {
  const double *ap, *bp;  // PACK_FRAG64 panels, Mpad / Npad multiples of 128
  long kq;                // Kpad / 4
  double *c;
  long rs_c, cs_c;
  int m, n, k;
  int tiles_m, tiles_n;
  const int2 *tile_list;  // (tm, tn) of the tiles to compute, or null: all tiles
  int ntiles;             // entries of tile_list
  double alpha, beta;
  int jp, ji, pi;
  int *err;
  unsigned long long wait_ns;  // bound of every mbarrier wait
  int stall;                   // failure-detection test: the producer issues no loads
  // Split-K: each tile's k range in `splits` chunks (units tile * splits +
  // chunk, taken round-robin by the persistent CTAs); with splits > 1 every
  // chunk stores its sums in `partials` and the last of a tile's chunks to
  // finish (counted in `arrivals`, zeroed) adds them in chunk order.
  int splits = 1;
  int *arrivals = nullptr;
  double *partials = nullptr;
  // Direct operand loads (no pack pass): 2-D TMA tiles read straight from
  // the caller's op(A) and op(B), one tensor map per operand and pair (a
  // SYR2K's two pairs split k at kpair, a multiple of the k-block).
  // a_kcontig / b_kcontig: the operand's unit stride runs along k (tiles
  // then land 128-byte swizzled, k innermost); otherwise along m / n.
  int direct = 0;
  int a_kcontig = 0, b_kcontig = 0;
  int npairs = 1;
  long kpair = 0;
  CUtensorMap ta[2], tb[2];
};
int launch_dmma_gemm(const DmmaGemmArgs &a, cudaStream_t s);
constexpr int B200_DMMA_TILE = 128, B200_DMMA_BK = 16;

template <typename T>
struct SimtConfig;

template <>
struct SimtConfig<float> {
  static constexpr int BM = 128, BN = 128, BK = 16;  // panel padding (tiles may be smaller)
};
template <>
struct SimtConfig<double> {
  static constexpr int BM = 128, BN = 128, BK = 16;  // panel padding (tiles may be smaller)
};

// pol == nullptr: one tile per CTA, no scratch (the allocation-free entry
// point); otherwise persistent CTAs with split-K and stream-ordered scratch.
template <typename T>
int launch_simt_gemm(const SimtGemmArgs<T> &a, cudaStream_t s, const SimtPolicy *pol = nullptr);

// ---- output-tile scheduling shared by the persistent GEMM kernels (sched.cu)

// The product's domain relations (mublis_l3_relation_t values).
struct b200_tile_domain_t {
  int jp, ji, pi;
};

// The BM x BN tiles of an m x n output that write under ji (the reference's
// block_is_outside, l3_driver.c:145-147,165-171), heaviest first (stable),
// as (tm, tn); costs, when given, receives each tile's k-blocks of BK after
// clipping its k range to jp / pi (l3_driver.c:130,148-150,163,171).
void b200_tile_list(long m, long n, long k, int BM, int BN, int BK, b200_tile_domain_t dom,
                    std::vector<int2> *list, std::vector<int> *costs);

// Split-K factor for a whole call (m_full x n_full x k) on `slots` resident
// persistent CTAs that take units (tile, k-chunk) heaviest tile first: the
// S in 1..16 (chunks of at least 8 k-blocks) whose simulated list schedule
// ends first, counting a fixed start-up cost per unit and split_cost
// (k-block times) more per split unit; S > 1 is taken only when it beats
// S = 1 by 10%.  Depends only on its arguments (cached per shape), so every
// column panel of a call splits its tiles as the whole call does.
int b200_split_for(long m_full, long n_full, long k, int BM, int BN, int BK,
                   b200_tile_domain_t dom, long slots, double split_cost);

template <typename T>
int launch_scale(int m, int n, T beta, T *c, long rs, long cs, int ji, cudaStream_t s);
