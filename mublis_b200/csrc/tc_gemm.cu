// tc_gemm.cu -- tcgen05 contraction forms (placeholder until the kernels land).
#include "tc_gemm.cuh"

int tc_run_bf16(const b200_l3_desc_t *, int) {
  return b200_set_error(B200_EINVAL, "bf16 split form not available in this build");
}
int tc_run_ozaki(const b200_l3_desc_t *) {
  return b200_set_error(B200_EINVAL, "ozaki form not available in this build");
}
