/*
 * b200_internal.h -- C-ABI between the C host layer (cblas, BLAS shims,
 * driver front-end, context) and the CUDA side of libmublis.
 *
 * Everything below takes DEVICE pointers: the host layer resolves caller
 * memory (host buffers are staged, device buffers are used in place) before
 * calling in.  All work is issued on the calling thread's library stream;
 * b200_stream_sync() makes it visible.
 */
#ifndef MUBLIS_B200_INTERNAL_H
#define MUBLIS_B200_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#include "../../include/mublis.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
  B200_OK = 0,
  B200_EINVAL = 1, /* bad argument or unsupported request */
  B200_ECUDA = 2,  /* a CUDA call failed (no device, launch error, ...) */
  B200_ENOMEM = 3, /* device or pinned allocation failed, or admission refused */
  B200_ETIMEOUT = 4 /* a bounded device-side wait gave up */
};

enum { B200_F32 = 0, B200_F64 = 1 };

/* Arithmetic form of the contraction.  PLAIN: FP32/FP64 FMA pipes.
 * BF16X3: FP32 operands split into bf16 hi+lo, three tcgen05 products per
 * k-block accumulated in FP32 (hi*hi + hi*lo + lo*hi).  BF16X6: three-term
 * split, six products.  OZAKI: FP64 via int8 slices with exact int32
 * accumulation (slice count in `slices`).  OZAKI2: FP64 via int8 residues
 * modulo N coprime moduli, one exact int8 product per modulus and a CRT
 * reconstruction (N in `slices`). */
enum { B200_FORM_AUTO = -1, B200_FORM_PLAIN = 0, B200_FORM_BF16X3 = 1, B200_FORM_BF16X6 = 2,
       B200_FORM_OZAKI = 3, B200_FORM_POLICY = 4 /* "auto": per-call size crossover */,
       B200_FORM_OZAKI2 = 5, B200_FORM_FP16X3 = 6 /* FP32 via scaled fp16 hi/lo, 3 products */ };

/* Parse a form name ("plain", "bf16x3", "bf16x6", "fp16x3", "ozaki[:s]",
 * "ozaki2[:N]", "ozaki2@<target error>", "auto"); B200_FORM_AUTO for
 * anything else.  *slices gets s or N, *target the error target, when given
 * (either may be NULL). */
int b200_parse_form(const char *s, int *slices, double *target);
/* The "ozaki2@<target>" error target of a precision's default form (0:
 * none). */
double b200_get_default_target(int dtype);

/* Loads the tuned-tile table named by MUBLIS_B200_TUNE_FILE, if any (called
 * once at initialisation). */
void b200_tune_autoload(void);

/* One product C(ji) := alpha * sum_t A_t B_t + beta * C over the domain of
 * `product`.  npairs is 1, or 2 for SYR2K (both pairs share the product's
 * operand structure and are concatenated along k). */
typedef struct {
  int dtype;
  int m, n, k;
  double alpha, beta;
  int npairs;
  const void *a[2];
  long rs_a[2], cs_a[2];
  const void *b[2];
  long rs_b[2], cs_b[2];
  void *c;
  long rs_c, cs_c;
  mublis_l3_product_t product;
  int form;   /* B200_FORM_* or AUTO (library default for the dtype) */
  int slices; /* Ozaki slice count, 0 = library default */
  long policy_n; /* n the "auto" policy decides on (0: n).  A column panel of a
                  * larger call carries the call's n, so every panel takes the
                  * form the whole call would. */
  long policy_m; /* same for m (0: m): triangle panels cover fewer rows */
} b200_l3_desc_t;

/* Left-side solve op(A) X = alpha B, already normalised by the host layer
 * (side RIGHT and trans folded into strides/uplo as trsm.c:35-54 does). */
typedef struct {
  int dtype;
  int m, n;
  double alpha;
  const void *a;
  long rs_a, cs_a;
  void *b;
  long rs_b, cs_b;
  mublis_uplo_t uplo; /* LOWER or UPPER of op(A) */
  int unit_diag;
  int form;
  int slices;
  long policy_n; /* as in b200_l3_desc_t, passed to the update products */
  const void *prep; /* diagonal inverses from b200_trsm_prepare, or NULL */
} b200_trsm_desc_t;

/* trsm.cu: the inverted diagonal blocks depend only on A, so a solve split
 * into column panels builds them once (prepare, on the calling thread's
 * stream), passes the result in each panel's desc (prep) and releases it
 * after the last panel. */
int b200_trsm_prepare(const b200_trsm_desc_t *d, void **prep);
void b200_trsm_release(void *prep);

/* trsm_leaf.cu: the fused GEMMTRSM kernel on leaves of b200_trsm_leaf_rows()
 * rows.  pack: every leaf of op(A) (order m; lower, or upper read reversed)
 * into leaves * b200_trsm_leaf_stride() elements; solve: one leaf of `rows`
 * rows for n right-hand sides, b at the leaf's first row in lower
 * orientation (an upper leaf: its last row, rs_b negated). */
long b200_trsm_leaf_rows(void);
long b200_trsm_leaf_stride(void);
int b200_trsm_leaf_pack(int dtype, const void *a, long rs_a, long cs_a, int m, int lower,
                        int unit, void *out);
int b200_trsm_leaf_solve(int dtype, const void *pack, int rows, void *b, long rs_b, long cs_b,
                         int n);

/* runtime.cu */
int b200_init(void);
int b200_device_count(void);
int b200_is_device_ptr(const void *p);
void *b200_stream(void);
int b200_set_thread_stream(void *stream);
/* Makes `stream` the one b200_stream() returns on this thread (nullptr:
 * back to the thread's own) and returns the previous override. */
void *b200_override_stream(void *stream);
/* A second stream paired with the calling thread's current stream, created
 * on first use (nullptr when none can be had). */
void *b200_aux_stream(void);
int b200_stream_sync(void);
int b200_alloc(void **p, size_t bytes);
void b200_free(void *p);
int b200_set_error(int code, const char *where);
/* Multiprocessor count of the calling thread's current device (cached). */
int b200_sm_count(void);
const char *b200_last_error(void);
int b200_get_default_form(int dtype);
int b200_set_default_form(int dtype, int form, int slices);
int b200_get_default_slices(int dtype);

/* Strided copies between caller host memory and a compact device buffer of
 * rows x cols with leading dimension ld (column-major).  The host side may
 * have any (rs, cs). */
/* Column-panel pipeline for host-resident operands.  The output (and an
 * optional input with the same columns) are moved in panels of columns:
 * panel J's host->device copy, its computation and panel J-1's copy back run
 * on three streams at once (PCIe is full duplex), so the transfers of a
 * large call overlap its own arithmetic.  `run` computes one panel on the
 * calling thread's library stream.  A view can be moved by panels when one
 * of its strides is 1 (b200_colpipe_view_ok). */
typedef struct {
  const void *host; /* NULL: no such operand */
  long rows, rs, cs;
} b200_colpipe_view_t;
/* An operand moved in index blocks beside the panels: with panel
 * [j0, j0 + cols), rows (by_cols = 0) or columns (by_cols = 1) j0 .. j0 +
 * cols - 1 of the host view, all `extent` elements of the other dimension,
 * go to the same indices of its whole device copy.  Host and device agree
 * on the unit stride (rs == drs == 1 or cs == dcs == 1). */
typedef struct {
  const void *host;
  long rs, cs;
  void *dev;
  long drs, dcs;
  long extent;
  int by_cols;
} b200_colpipe_stream_t;
enum { B200_COLPIPE_MAX_PANELS = 8, B200_COLPIPE_MAX_STREAMS = 4 };
typedef struct {
  size_t elt;
  long ncols;
  b200_colpipe_view_t in;  /* read-only input panel (op(B)), or host NULL */
  b200_colpipe_view_t out; /* output panel (C, or B in place) */
  int out_read;            /* copy the output panel in before computing */
  int (*run)(void *ctx, long j0, long cols, void *in_dev, long in_rs, long in_cs,
             void *out_dev, long out_rs, long out_cs);
  void *ctx;
  long panel_min; /* narrowest panel worth computing (0: 1024 columns) */
  int out_lower;  /* the output is a lower triangle: panel j0 moves only rows
                     j0.. (out_dev is then element (j0, j0)); needs out_read */
  int nwidths;    /* > 0: explicit panel widths, left to right (else even panels) */
  long widths[B200_COLPIPE_MAX_PANELS];
  int reverse;    /* compute the panels right to left */
  int nstreams;
  b200_colpipe_stream_t streams[B200_COLPIPE_MAX_STREAMS];
} b200_colpipe_t;
int b200_colpipe_view_ok(long rows, long rs, long cs);
/* Number of panels worth using for ncols columns of total bytes (< 2: do
 * not pipeline). */
int b200_colpipe_panels(long ncols, size_t bytes);
/* Same with panels of at least min_cols columns. */
int b200_colpipe_panels_min(long ncols, size_t bytes, long min_cols);
int b200_column_pipeline(const b200_colpipe_t *p);

#ifdef __CUDACC__
/* Host-to-device 2-D copy on s; large ones split over two copy engines. */
cudaError_t b200_h2d_2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
                        size_t height, cudaStream_t s);
#endif
int b200_copy_h2d(void *dst, long ld, const void *src, long rs, long cs, long rows, long cols,
                  size_t elt);
int b200_copy_d2h(void *dst, long rs, long cs, const void *src, long ld, long rows, long cols,
                  size_t elt);

/* runtime.cu: the wait limit armed by mublis_b200_test_stall_next (0 when
 * none is armed), cleared by the call: the next FP64 tensor-pipe GEMM launch
 * takes it and stalls. */
unsigned long long b200_take_test_stall(void);

/* noalloc.cu: resolves the allocation-free SGEMM's fixed scratch array on
 * the current device (run once by b200_init). */
void b200_noalloc_setup(void);

/* tc_gemm.cu: nonzero (and cleared) if a kernel reported a bounded-wait
 * timeout since the last call. */
int b200_take_device_error(void);

/* l3.cu */
int b200_l3_run(const b200_l3_desc_t *d);
int b200_trsm_run(const b200_trsm_desc_t *d);
int b200_scale_strided(int dtype, int m, int n, double beta, void *c, long rs, long cs,
                       mublis_l3_relation_t ji);

/* grouped.cu: asynchronous batched execution on `stream` (the request
 * server's coalesced launches).  Every descriptor must be batchable: a
 * plain GEMM (general operands, domain ALL, one pair) of the given dtype, or
 * a left TRSM of order <= 256 with alpha != 0. */
int b200_l3_is_plain_gemm(const b200_l3_desc_t *d);
int b200_grouped_gemm_async(int dtype, const b200_l3_desc_t *const *descs, int count,
                            void *stream);
int b200_grouped_trsm_async(int dtype, const b200_trsm_desc_t *const *descs, int count,
                            void *stream);
/* One plain GEMM read directly from its operands (no pack pass, no scratch),
 * on the calling thread's stream. */
int b200_gemm_direct(const b200_l3_desc_t *d);
/* Same, with tiles at least min_rows tall (for in-place products). */
int b200_gemm_direct_min_rows(const b200_l3_desc_t *d, int min_rows);

/* serve.cu: when a request server is attached, the host front routes calls
 * whose operands are all device-resident through it (blocking until done).
 * b200_serve_attached() is 0 when none is attached. */
int b200_serve_attached(void);
int b200_serve_l3(const b200_l3_desc_t *d);
int b200_serve_trsm(const b200_trsm_desc_t *d);

/* ukr.cu: one MR x NR micro-tile on the device (packed host panels). */
int b200_ukr_gemm(int dtype, int k, const void *alpha, const void *a, const void *b,
                  const void *beta, void *c, int rs_c, int cs_c, int mr, int nr);
int b200_ukr_gemmtrsm(int dtype, int lower, int k, const void *alpha, const void *a1x,
                      const void *a11, const void *bx1, void *b11, void *c11, int rs_c,
                      int cs_c, int mr, int nr);

#ifdef __cplusplus
}
#endif

#endif
