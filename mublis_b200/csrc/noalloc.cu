// noalloc.cu -- an SGEMM entry point that allocates no memory.
//
// Some callers cannot allocate device memory at the moment they call into
// the library: a process whose GPU memory is already fully claimed by
// another allocator (for example a framework's caching allocator that has
// reserved the device), or a service that must keep a fixed device-memory
// footprint once it is running and therefore forbids cudaMalloc / cudaFree
// on its request path.  mublis_b200_sgemm_noalloc serves them: it computes
// exactly what mublis_sgemm computes on device operands (same pack pass,
// same plain FP32 kernel), but stages the packed operand panels in a fixed
// scratch array that is part of the library's device image instead of in
// memory allocated per call.
//
// The array, g_noalloc_scratch, holds NOALLOC_SCRATCH_FLOATS floats
// (32 MiB).  In host code its name is only a host-side stand-in for the
// device symbol, so the device address is obtained once per device, with
// that device current, through cudaGetSymbolAddress.  That lookup is also
// what loads this file's device code (CUDA loads modules lazily) and with it
// claims the 32 MiB, which the device then keeps until the process exits.
// The library's initialisation (b200_init, run by mublis_b200_init or the
// first call of any entry point) does it for the device current at that
// moment, so the memory is claimed when the library starts, not on a
// request path; on any other device the first call of this entry point
// there does it.
//
// Every call on a device shares the one array, and the array keeps whatever
// the last call left in it.  Nothing in it needs to start at zero: the pack
// pass rewrites every element of the padded panels the kernel will read,
// padding included.  Calls that overlap on the GPU (for example two host
// threads calling at once on the same device) race on the array; callers
// must not overlap them.
#include <cstdio>
#include <mutex>

#include "kernels.cuh"
#include "../../include/mublis_b200.h"

#define NOALLOC_SCRATCH_FLOATS (8L << 20) /* 32 MiB of FP32 */

static __device__ __align__(256) float g_noalloc_scratch[NOALLOC_SCRATCH_FLOATS];

namespace {

constexpr int NOALLOC_MAX_DEVICES = 64;

float *g_scratch_addr[NOALLOC_MAX_DEVICES];
int g_scratch_status[NOALLOC_MAX_DEVICES];
std::once_flag g_scratch_once[NOALLOC_MAX_DEVICES];

// Device address of g_noalloc_scratch on the current device (looked up
// once per device).
int scratch_on_current_device(float **out) {
  int dev = 0;
  B200_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return b200_set_error(B200_EINVAL, "sgemm_noalloc: device index out of range");
  std::call_once(g_scratch_once[dev], [dev] {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      b200_note_cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
      g_scratch_status[dev] = B200_ECUDA;
      return;
    }
    g_scratch_addr[dev] = static_cast<float *>(p);
    g_scratch_status[dev] = B200_OK;
  });
  if (g_scratch_status[dev] != B200_OK)
    return b200_set_error(g_scratch_status[dev],
                          "sgemm_noalloc: could not resolve the scratch array on this device");
  *out = g_scratch_addr[dev];
  return B200_OK;
}

}  // namespace

// Called once by the library's initialisation with the device it brings up
// current: resolves (and so claims) the scratch array there.  A failure is
// kept and reported by the entry point's first call; it does not fail the
// initialisation of everything else.
extern "C" void b200_noalloc_setup(void) {
  float *unused = nullptr;
  (void)scratch_on_current_device(&unused);
}

extern "C" int mublis_b200_sgemm_noalloc(mublis_trans_t trans_a, mublis_trans_t trans_b, int m,
                                         int n, int k, float alpha, const float *a, int rs_a,
                                         int cs_a, const float *b, int rs_b, int cs_b, float beta,
                                         float *c, int rs_c, int cs_c) {
  // Same order of checks as mublis_sgemm: an empty output returns before
  // the sizes are checked.
  if (m == 0 || n == 0) return B200_OK;
  if (m < 0 || n < 0 || k < 0) return b200_set_error(B200_EINVAL, "sgemm_noalloc: negative size");
  B200_TRY(b200_init());
  const bool update = alpha != 0.f && k > 0;
  if (!b200_is_device_ptr(c) || (update && (!b200_is_device_ptr(a) || !b200_is_device_ptr(b))))
    return b200_set_error(B200_EINVAL,
                          "sgemm_noalloc: A, B and C must be device pointers (staging host "
                          "operands would allocate)");
  cudaStream_t s = b200_cur_stream();
  if (!update) {
    B200_TRY(launch_scale<float>(m, n, beta, c, rs_c, cs_c, MUBLIS_L3_ALL, s));
    return b200_stream_sync();
  }

  using Cfg = SimtConfig<float>;
  const long mpad = b200_round_up(m, Cfg::BM), npad = b200_round_up(n, Cfg::BN);
  const long kpad = b200_round_up(k, Cfg::BK);
  if ((mpad + npad) * kpad > NOALLOC_SCRATCH_FLOATS) {
    char msg[256];
    snprintf(msg, sizeof msg,
             "sgemm_noalloc: m=%d n=%d k=%d needs %ld scratch floats "
             "((roundup(m,%d) + roundup(n,%d)) * roundup(k,%d)); the maximum is %ld",
             m, n, k, (mpad + npad) * kpad, Cfg::BM, Cfg::BN, Cfg::BK, NOALLOC_SCRATCH_FLOATS);
    return b200_set_error(B200_EINVAL, msg);
  }
  float *scratch = nullptr;
  B200_TRY(scratch_on_current_device(&scratch));
  float *ap = scratch, *bp = scratch + mpad * kpad;

  // op() as a stride swap, exactly as the BLAS mirror does (frame/l3/gemm.c:14-24).
  long ars = rs_a, acs = cs_a, brs = rs_b, bcs = cs_b;
  if (trans_a == MUBLIS_TRANSPOSE) { long t = ars; ars = acs; acs = t; }
  if (trans_b == MUBLIS_TRANSPOSE) { long t = brs; brs = bcs; bcs = t; }
  PackView va{a, ars, acs, MUBLIS_STRUC_GENERAL, MUBLIS_DENSE, MUBLIS_PACKM_DIAG_NONUNIT,
              MUBLIS_L3_ALL};
  PackView vb{b, brs, bcs, MUBLIS_STRUC_GENERAL, MUBLIS_DENSE, MUBLIS_PACKM_DIAG_NONUNIT,
              MUBLIS_L3_ALL};
  PackOut oa{ap, mpad, 0, PACK_MN_MAJOR, PACK_COPY, 1, nullptr};
  PackOut ob{bp, npad, 0, PACK_MN_MAJOR, PACK_COPY, 1, nullptr};
  B200_TRY(launch_pack<float>(va, false, m, k, mpad, 0, kpad, oa, s));
  B200_TRY(launch_pack<float>(vb, true, n, k, npad, 0, kpad, ob, s));

  SimtGemmArgs<float> g;
  g.ap = ap;
  g.bp = bp;
  g.lda = mpad;
  g.ldb = npad;
  g.c = c;
  g.rs_c = rs_c;
  g.cs_c = cs_c;
  g.m = m;
  g.n = n;
  g.k = k;
  g.alpha = alpha;
  g.beta = beta;
  g.jp = g.ji = g.pi = MUBLIS_L3_ALL;
  B200_TRY(launch_simt_gemm<float>(g, s));
  return b200_stream_sync();
}
