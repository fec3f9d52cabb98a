// common.cuh -- shared device/host helpers for the CUDA side of libmublis.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "b200_internal.h"

#define B200_CUDA_TRY(expr)                                                   \
  do {                                                                        \
    cudaError_t b200_err_ = (expr);                                           \
    if (b200_err_ != cudaSuccess) {                                           \
      b200_note_cuda_error(b200_err_, #expr, __FILE__, __LINE__);             \
      return b200_err_ == cudaErrorMemoryAllocation ? B200_ENOMEM : B200_ECUDA; \
    }                                                                         \
  } while (0)

#define B200_TRY(expr)                 \
  do {                                 \
    int b200_st_ = (expr);             \
    if (b200_st_ != B200_OK) return b200_st_; \
  } while (0)

// Records a CUDA failure as the thread's last error (string) and returns it.
void b200_note_cuda_error(cudaError_t err, const char *what, const char *file, int line);

static inline cudaStream_t b200_cur_stream() { return (cudaStream_t)b200_stream(); }

// Launch-error check after a kernel launch.
#define B200_LAUNCH_CHECK() B200_CUDA_TRY(cudaGetLastError())

// Per-kernel timing (enabled by mublis_b200_profile_enable): brackets a
// launch with CUDA events on the launching stream.
struct B200ProfScope {
  int slot;
  cudaStream_t stream;
  B200ProfScope(const char *name, cudaStream_t s);
  ~B200ProfScope();
};

// Runs `setup` once per process: callers that arrive while it runs wait for
// it, and every caller gets its status (with a last-error message of its own
// when it failed: `what`).  For one-time kernel attribute set-up that several
// host threads may reach first at the same time.
template <class F>
int b200_once(std::once_flag &flag, int &status, const char *what, F setup) {
  std::call_once(flag, [&] { status = setup(); });
  return status == B200_OK ? B200_OK : b200_set_error(status, what);
}

static inline long b200_round_up(long x, long m) { return (x + m - 1) / m * m; }
static inline long b200_ceil_div(long x, long m) { return (x + m - 1) / m; }

// Relation test of frame/l3/l3_utils.c:18-28 (LOWER: lhs <= rhs, UPPER:
// lhs >= rhs), usable on both sides.
__host__ __device__ static inline bool b200_rel(int rel, long lhs, long rhs) {
  return rel == MUBLIS_L3_LOWER ? lhs <= rhs : (rel == MUBLIS_L3_UPPER ? lhs >= rhs : true);
}
