// tc_gemm.cuh -- tcgen05 (5th-generation tensor core) forms of the L3
// contraction: BF16x3 / BF16x6 split FP32 and Ozaki int8-sliced FP64.
#pragma once

#include "common.cuh"

int tc_run_bf16(const b200_l3_desc_t *d, int form);
int tc_run_ozaki(const b200_l3_desc_t *d);
