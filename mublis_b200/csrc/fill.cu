// fill.cu -- seeded device fills (Philox4x32-10, Salmon et al. SC'11).
//
// Key = (seed, matrix_id), counter = (idx_lo, idx_hi, 0, 0) with idx the
// column-major element index i + j*m.  The draws are defined so the device
// values are bit-identical to a host implementation of the same algorithm:
//   uniform f32 : (w0 >> 8) * 2^-23 - 1          f64 : (w0:w1 >> 11) * 2^-52 - 1
//   wide        : +-(1 + frac) * 2^e, frac from w0 (f32: w0 >> 9; f64: 52 bits of
//                 w0:w1), e = w3 % 21 - 10, sign = w2 & 1
//   diag        : 1 + (uniform + 1) / 2           (in [1, 2))
#include "common.cuh"
#include "../../include/mublis_b200.h"

namespace {

__device__ __forceinline__ uint4 philox4x32_10(unsigned long long index, uint32_t seed,
                                               uint32_t id) {
  uint32_t c0 = (uint32_t)index, c1 = (uint32_t)(index >> 32), c2 = 0, c3 = 0;
  uint32_t k0 = seed, k1 = id;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
    uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return make_uint4(c0, c1, c2, c3);
}

__device__ __forceinline__ float draw_f32(unsigned long long idx, uint32_t seed, uint32_t id,
                                          int kind) {
  uint4 w = philox4x32_10(idx, seed, id);
  float u = __fsub_rn(__fmul_rn((float)(w.x >> 8), 0x1p-23f), 1.0f);
  if (kind == 2) return __fadd_rn(1.0f, __fmul_rn(__fadd_rn(u, 1.0f), 0.5f));
  if (kind == 1) {
    float mant = __fadd_rn(1.0f, __fmul_rn((float)(w.x >> 9), 0x1p-23f));
    int e = (int)(w.w % 21u) - 10;
    float x = ldexpf(mant, e);
    return (w.z & 1u) ? -x : x;
  }
  return u;
}

__device__ __forceinline__ double draw_f64(unsigned long long idx, uint32_t seed, uint32_t id,
                                           int kind) {
  uint4 w = philox4x32_10(idx, seed, id);
  unsigned long long bits = (((unsigned long long)w.x << 32) | w.y) >> 11;
  double u = __dsub_rn(__dmul_rn((double)bits, 0x1p-52), 1.0);
  if (kind == 2) return __dadd_rn(1.0, __dmul_rn(__dadd_rn(u, 1.0), 0.5));
  if (kind == 1) {
    double mant = __dadd_rn(1.0, __dmul_rn((double)(bits >> 1), 0x1p-52));
    int e = (int)(w.w % 21u) - 10;
    double x = ldexp(mant, e);
    return (w.z & 1u) ? -x : x;
  }
  return u;
}

template <typename T>
__global__ void fill_kernel(T *x, long m, long n, long ld, uint32_t seed, uint32_t id, int kind) {
  long total = m * n;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    long i = t % m, j = t / m;
    T v;
    if (sizeof(T) == 4) v = (T)draw_f32((unsigned long long)t, seed, id, kind);
    else v = (T)draw_f64((unsigned long long)t, seed, id, kind);
    x[i + j * ld] = v;
  }
}

template <typename T>
int fill(T *x, long m, long n, long ld, uint32_t seed, uint32_t id, int kind) {
  B200_TRY(b200_init());
  if (m <= 0 || n <= 0) return B200_OK;
  if (ld < m || kind < 0 || kind > 2) return b200_set_error(B200_EINVAL, "fill: bad arguments");
  cudaStream_t s = b200_cur_stream();
  long blocks = std::min<long>(b200_ceil_div(m * n, 256), 148L * 32);
  {
    B200ProfScope prof("fill", s);
    fill_kernel<T><<<(unsigned)blocks, 256, 0, s>>>(x, m, n, ld, seed, id, kind);
    B200_LAUNCH_CHECK();
  }
  return b200_stream_sync();
}

}  // namespace

extern "C" int mublis_b200_fill_s(float *x, long m, long n, long ld, uint32_t seed,
                                  uint32_t matrix_id, int kind) {
  return fill<float>(x, m, n, ld, seed, matrix_id, kind);
}
extern "C" int mublis_b200_fill_d(double *x, long m, long n, long ld, uint32_t seed,
                                  uint32_t matrix_id, int kind) {
  return fill<double>(x, m, n, ld, seed, matrix_id, kind);
}
