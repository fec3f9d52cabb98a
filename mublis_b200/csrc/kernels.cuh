// kernels.cuh -- launchers shared between the CUDA translation units.
#pragma once

#include <cuda_bf16.h>

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

// Output orientation of a packed panel.  The panel covers mn in [0, mn_pad)
// and kk in [kk0, kk1); logical element (mn, kk - kk0) is taken from the
// view, as (r, c) = (mn, kk) for an A-side view or (kk, mn) for a B-side
// view; anything past mn_len / k_len is zero.
enum PackLayout {
  PACK_MN_MAJOR = 0,  // out[kk * ld + mn]       (SIMT kernels)
  PACK_K_MAJOR = 1    // out[mn * ld + kk]       (tcgen05 kernels)
};

enum PackXform {
  PACK_COPY = 0,        // T -> T
  PACK_BF16_SPLIT = 1,  // f32 -> `terms` bf16 planes (hi, lo[, lo2])
  PACK_INT8_SLICES = 2  // f64 -> `terms` int8 planes of 7-bit slices of
                        // x * 2^(7 - e), e from the row/column abs-max
};

struct PackOut {
  void *out;
  long ld;
  long plane_stride;  // elements between planes
  int layout, xform, terms;
  const unsigned long long *absmax;  // PACK_INT8_SLICES: bits of max |x| per mn
};

// Bits of max |x| over kk for every mn of a logical operand view (the
// Ozaki split's per-row / per-column scale), atomically max-merged into
// absmax[mn] (which must start at 0).
int launch_absmax(const PackView &v, bool b_side, long mn_len, long k_len,
                  unsigned long long *absmax, cudaStream_t s);

// Exponent e with max|x| < 2^e (frexp), 0 for an all-zero row.
__device__ inline int b200_scale_exp(unsigned long long absmax_bits) {
  if (absmax_bits == 0) return 0;
  int e;
  frexp(__longlong_as_double((long long)absmax_bits), &e);
  return e;
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
};

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

template <typename T>
int launch_simt_gemm(const SimtGemmArgs<T> &a, cudaStream_t s);

template <typename T>
int launch_scale(int m, int n, T beta, T *c, long rs, long cs, int ji, cudaStream_t s);
