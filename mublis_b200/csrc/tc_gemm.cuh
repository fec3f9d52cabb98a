// tc_gemm.cuh -- tcgen05 (5th-generation tensor core) forms of the L3
// contraction: BF16x3 / BF16x6 split FP32 and Ozaki int8-sliced FP64.
#pragma once

#include "common.cuh"

int tc_run_bf16(const b200_l3_desc_t *d, int form);
int tc_run_ozaki(const b200_l3_desc_t *d);

#include "../../include/mublis_b200.h"

// tc_grouped.cu: a group of FP32 GEMMs in the fp16x3 form.  create builds
// the device tables and staging areas (synchronous; not during capture),
// run launches the pack and the tensor-core kernel on `s` (capturable),
// destroy frees them.
struct b200_tcg;
int b200_tcg_create(const mublis_b200_gemm_problem_t *p, int count, b200_tcg **out);
int b200_tcg_run(b200_tcg *g, cudaStream_t s);
void b200_tcg_destroy(b200_tcg *g);

#include <string>

// ozaki_tune.cu: the modulus count of the modular form for a target
// normwise error, measured on a calibration block of the call (cached per
// precision, k bucket and target; force = 1 measures again).
int b200_ozaki2_choice(const b200_l3_desc_t *d, double target, int *moduli, double *measured,
                       int force);
// Tuned-table persistence of those choices (lines appended / parsed by the
// table's save and load; reset clears them).
void b200_ozaki2_table_lines(std::string *text);
bool b200_ozaki2_table_parse(const char *line);
void b200_ozaki2_table_reset();
// grouped.cu: rewrites the table named by MUBLIS_B200_TUNE_FILE, if any.
void b200_tune_save_env();
