// ukr.cu -- device-backed micro-kernels behind b200_context.
//
// They honour the packed-panel ABI of include/mublis_instantiate.h
// (gemm_ukr :37-52, gemmtrsm_ukr :71-94): the caller passes HOST panels
// (A(i,p) = a[p*MR+i], B(p,j) = b[p*NR+j]); one MR x NR tile is computed on
// the GPU and written back through (rs_c, cs_c).  They are the contract
// surface for code that drives its own loops; the library's routines do not
// call them (they tile whole problems on the device, l3.cu).
#include <vector>

#include "common.cuh"

namespace {

template <typename T>
__global__ void ukr_gemm_kernel(int k, T alpha, const T *a, const T *b, T beta, T *c, int mr,
                                int nr) {
  int i = threadIdx.x, j = blockIdx.x;
  if (i >= mr || j >= nr) return;
  T s = T(0);
  for (int p = 0; p < k; ++p) s = fma(a[p * mr + i], b[p * nr + j], s);
  T v = alpha * s;
  if (beta != T(0)) v = fma(beta, c[i + j * mr], v);
  c[i + j * mr] = v;
}

// One thread per right-hand-side column; A11 is column-major mr x mr with
// its diagonal already inverted.
template <typename T>
__global__ void ukr_gemmtrsm_kernel(bool lower, int k, T alpha, const T *a1x, const T *a11,
                                    const T *bx1, T *b11, int mr, int nr) {
  int j = threadIdx.x;
  if (j >= nr) return;
  for (int q = 0; q < mr; ++q) {
    int i = lower ? q : mr - 1 - q;
    T r = alpha * b11[i * nr + j];
    for (int p = 0; p < k; ++p) r = fma(-a1x[p * mr + i], bx1[p * nr + j], r);
    if (lower)
      for (int p = 0; p < i; ++p) r = fma(-a11[i + p * mr], b11[p * nr + j], r);
    else
      for (int p = i + 1; p < mr; ++p) r = fma(-a11[i + p * mr], b11[p * nr + j], r);
    b11[i * nr + j] = r * a11[i + i * mr];
  }
}

template <typename T>
int run_gemm(int k, T alpha, const T *a, const T *b, T beta, T *c, int rs_c, int cs_c, int mr,
             int nr) {
  B200_TRY(b200_init());
  if (mr > 1024 || nr > 65535) return b200_set_error(B200_EINVAL, "ukr tile too large");
  cudaStream_t s = b200_cur_stream();
  std::vector<T> tile((size_t)mr * nr);
  if (beta != T(0))
    for (int j = 0; j < nr; ++j)
      for (int i = 0; i < mr; ++i) tile[i + (size_t)j * mr] = c[i * rs_c + j * cs_c];
  T *da = nullptr, *db = nullptr, *dc = nullptr;
  size_t ka = (size_t)(k > 0 ? k : 1);
  B200_TRY(b200_alloc((void **)&da, sizeof(T) * ka * mr));
  B200_TRY(b200_alloc((void **)&db, sizeof(T) * ka * nr));
  B200_TRY(b200_alloc((void **)&dc, sizeof(T) * mr * nr));
  if (k > 0) {
    B200_CUDA_TRY(cudaMemcpyAsync(da, a, sizeof(T) * k * mr, cudaMemcpyHostToDevice, s));
    B200_CUDA_TRY(cudaMemcpyAsync(db, b, sizeof(T) * k * nr, cudaMemcpyHostToDevice, s));
  }
  B200_CUDA_TRY(cudaMemcpyAsync(dc, tile.data(), sizeof(T) * mr * nr, cudaMemcpyHostToDevice, s));
  {
    B200ProfScope prof("ukr_gemm", s);
    ukr_gemm_kernel<T><<<nr, mr, 0, s>>>(k, alpha, da, db, beta, dc, mr, nr);
    B200_LAUNCH_CHECK();
  }
  B200_CUDA_TRY(cudaMemcpyAsync(tile.data(), dc, sizeof(T) * mr * nr, cudaMemcpyDeviceToHost, s));
  b200_free(da);
  b200_free(db);
  b200_free(dc);
  B200_TRY(b200_stream_sync());
  for (int j = 0; j < nr; ++j)
    for (int i = 0; i < mr; ++i) c[i * rs_c + j * cs_c] = tile[i + (size_t)j * mr];
  return B200_OK;
}

template <typename T>
int run_gemmtrsm(bool lower, int k, T alpha, const T *a1x, const T *a11, const T *bx1, T *b11,
                 T *c11, int rs_c, int cs_c, int mr, int nr) {
  B200_TRY(b200_init());
  if (nr > 1024) return b200_set_error(B200_EINVAL, "ukr tile too large");
  cudaStream_t s = b200_cur_stream();
  size_t ka = (size_t)(k > 0 ? k : 1);
  T *d1x = nullptr, *d11 = nullptr, *dbx = nullptr, *db11 = nullptr;
  B200_TRY(b200_alloc((void **)&d1x, sizeof(T) * ka * mr));
  B200_TRY(b200_alloc((void **)&d11, sizeof(T) * mr * mr));
  B200_TRY(b200_alloc((void **)&dbx, sizeof(T) * ka * nr));
  B200_TRY(b200_alloc((void **)&db11, sizeof(T) * mr * nr));
  if (k > 0) {
    B200_CUDA_TRY(cudaMemcpyAsync(d1x, a1x, sizeof(T) * k * mr, cudaMemcpyHostToDevice, s));
    B200_CUDA_TRY(cudaMemcpyAsync(dbx, bx1, sizeof(T) * k * nr, cudaMemcpyHostToDevice, s));
  }
  B200_CUDA_TRY(cudaMemcpyAsync(d11, a11, sizeof(T) * mr * mr, cudaMemcpyHostToDevice, s));
  B200_CUDA_TRY(cudaMemcpyAsync(db11, b11, sizeof(T) * mr * nr, cudaMemcpyHostToDevice, s));
  {
    B200ProfScope prof("ukr_gemmtrsm", s);
    ukr_gemmtrsm_kernel<T><<<1, nr, 0, s>>>(lower, k, alpha, d1x, d11, dbx, db11, mr, nr);
    B200_LAUNCH_CHECK();
  }
  B200_CUDA_TRY(cudaMemcpyAsync(b11, db11, sizeof(T) * mr * nr, cudaMemcpyDeviceToHost, s));
  b200_free(d1x);
  b200_free(d11);
  b200_free(dbx);
  b200_free(db11);
  B200_TRY(b200_stream_sync());
  for (int j = 0; j < nr; ++j)
    for (int i = 0; i < mr; ++i) c11[i * rs_c + j * cs_c] = b11[i * nr + j];
  return B200_OK;
}

}  // namespace

extern "C" int b200_ukr_gemm(int dtype, int k, const void *alpha, const void *a, const void *b,
                             const void *beta, void *c, int rs_c, int cs_c, int mr, int nr) {
  if (dtype == B200_F32)
    return run_gemm<float>(k, *(const float *)alpha, (const float *)a, (const float *)b,
                           *(const float *)beta, (float *)c, rs_c, cs_c, mr, nr);
  return run_gemm<double>(k, *(const double *)alpha, (const double *)a, (const double *)b,
                          *(const double *)beta, (double *)c, rs_c, cs_c, mr, nr);
}

extern "C" int b200_ukr_gemmtrsm(int dtype, int lower, int k, const void *alpha, const void *a1x,
                                 const void *a11, const void *bx1, void *b11, void *c11,
                                 int rs_c, int cs_c, int mr, int nr) {
  if (dtype == B200_F32)
    return run_gemmtrsm<float>(lower != 0, k, *(const float *)alpha, (const float *)a1x,
                               (const float *)a11, (const float *)bx1, (float *)b11,
                               (float *)c11, rs_c, cs_c, mr, nr);
  return run_gemmtrsm<double>(lower != 0, k, *(const double *)alpha, (const double *)a1x,
                              (const double *)a11, (const double *)bx1, (double *)b11,
                              (double *)c11, rs_c, cs_c, mr, nr);
}
