/*
 * front.h -- host front-end shared by the driver and the BLAS mirrors.
 *
 * Resolves caller memory for one call: device pointers are used in place,
 * host pointers are staged into compact device copies (in the orientation
 * whose unit stride matches the caller's, so the copy is a 2-D memcpy) and
 * copied back for outputs.  The call then runs on the calling thread's
 * library stream and is synchronised before returning, which keeps the
 * reference's synchronous, thread-safe contract (frame/base/pool.c:4-10).
 */
#ifndef MUBLIS_B200_FRONT_H
#define MUBLIS_B200_FRONT_H

#include "../b200_internal.h"

typedef struct {
  void *ptr; /* device address of element (0, 0) */
  long rs, cs;
} b200_view_t;

typedef struct {
  const void *host;
  long rows, cols, rs, cs; /* staged footprint, host strides */
  int transposed;          /* staged as cols x rows (caller's cs == 1) */
  void *dev;
  long ld;
  int out;
  int tri; /* 0: the whole view; 1: only c <= r (lower); 2: only c >= r (upper) */
} b200_stage_t;

typedef struct {
  b200_stage_t st[8];
  int n;
  size_t elt;
} b200_stage_set_t;

void b200_stage_begin(b200_stage_set_t *ss, size_t elt);
/* View of rows x cols elements at p with strides (rs, cs).  copy_in = 0
 * allocates without reading the caller's values; out = 1 copies back at
 * b200_stage_end. */
int b200_stage_view(b200_stage_set_t *ss, const void *p, long rows, long cols, long rs, long cs,
                    int copy_in, int out, b200_view_t *v);
/* Same, for an operand of which the call reads (and, with out, writes) only
 * one triangle (tri: 1 = elements with column <= row, 2 = column >= row):
 * only that triangle crosses PCIe, in blocks of columns, both ways (the
 * blocks that straddle the diagonal carry some of the other triangle, so an
 * output staged this way must also be copied in).  The rest of the other
 * triangle of the device copy is left unset and never copied back. */
int b200_stage_view_tri(b200_stage_set_t *ss, const void *p, long rows, long cols, long rs,
                        long cs, int copy_in, int out, int tri, b200_view_t *v);
/* Copies outputs back (when status is OK), frees, synchronises. */
int b200_stage_end(b200_stage_set_t *ss, int status);

int b200_front_l3(b200_l3_desc_t *d);
int b200_front_trmm(int dtype, mublis_side_t side, mublis_uplo_t uplo, mublis_trans_t trans,
                    mublis_diag_t diag, int m, int n, double alpha, const void *a, int rs_a,
                    int cs_a, void *b, int rs_b, int cs_b);
int b200_front_trsm(int dtype, mublis_side_t side, mublis_uplo_t uplo, mublis_trans_t trans,
                    mublis_diag_t diag, int m, int n, double alpha, const void *a, int rs_a,
                    int cs_a, void *b, int rs_b, int cs_b);

#endif
