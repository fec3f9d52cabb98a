/*
 * front.c -- the host side of mublis_l3_{s,d}driver, TRMM and TRSM.
 *
 *   mublis_l3_{s,d}driver  include/mublis.h:65-83, reference
 *                          frame/l3/l3_driver.c:49-256: same arguments, same
 *                          m == 0 || n == 0 early return (:61-62), status 0 on
 *                          success.  The descriptor goes to the device driver
 *                          (l3.cu) instead of the CPU loop nest.
 *   TRMM front             frame/l3/trmm.c:44-85 (normalisation and product
 *                          descriptor), :138-144 (alpha == 0 zeroes B)
 *   TRSM front             frame/l3/trsm.c:24-54 (alpha == 0 zeroes B; right
 *                          side -> left; trans -> stride swap + flip_uplo)
 */
#include "front.h"

#include <string.h>

static int views_same(const b200_stage_t *s, const void *p, long rows, long cols, long rs,
                      long cs) {
  return s->host == p && s->rows == rows && s->cols == cols && s->rs == rs && s->cs == cs;
}

void b200_stage_begin(b200_stage_set_t *ss, size_t elt) {
  memset(ss, 0, sizeof *ss);
  ss->elt = elt;
}

/* Copies a staged view between host and device: the whole view, or the
 * blocks of TRI_BLOCK columns of the device-side orientation restricted to
 * the rows that hold the staged triangle. */
enum { TRI_BLOCK = 256 };

static int stage_copy(const b200_stage_t *s, size_t elt, int to_device) {
  /* Device orientation: column-major R x C with leading dimension ld. */
  const long R = s->transposed ? s->cols : s->rows, C = s->transposed ? s->rows : s->cols;
  const long hrs = s->transposed ? s->cs : s->rs, hcs = s->transposed ? s->rs : s->cs;
  int tri = s->tri;
  if (s->transposed && tri) tri = tri == 1 ? 2 : 1;
  const long bw = tri ? TRI_BLOCK : C;
  for (long j0 = 0; j0 < C; j0 += bw) {
    const long j1 = j0 + bw < C ? j0 + bw : C;
    long i0 = 0, i1 = R;
    if (tri == 1) i0 = j0 < R ? j0 : R; /* column <= row: rows from the block's first column */
    if (tri == 2) i1 = j1 < R ? j1 : R; /* column >= row: rows up to the block's last column */
    if (i1 <= i0) continue;
    char *dev = (char *)s->dev + (size_t)(i0 + j0 * s->ld) * elt;
    const char *host = (const char *)s->host + (i0 * hrs + j0 * hcs) * (long)elt;
    int st = to_device ? b200_copy_h2d(dev, s->ld, host, hrs, hcs, i1 - i0, j1 - j0, elt)
                       : b200_copy_d2h((void *)host, hrs, hcs, dev, s->ld, i1 - i0, j1 - j0, elt);
    if (st != B200_OK) return st;
  }
  return B200_OK;
}

int b200_stage_view(b200_stage_set_t *ss, const void *p, long rows, long cols, long rs, long cs,
                    int copy_in, int out, b200_view_t *v) {
  return b200_stage_view_tri(ss, p, rows, cols, rs, cs, copy_in, out, 0, v);
}

int b200_stage_view_tri(b200_stage_set_t *ss, const void *p, long rows, long cols, long rs,
                        long cs, int copy_in, int out, int tri, b200_view_t *v) {
  v->ptr = (void *)p;
  v->rs = rs;
  v->cs = cs;
  if (rows <= 0 || cols <= 0) return B200_OK;
  if (p == NULL) return b200_set_error(B200_EINVAL, "null operand pointer");
  if (b200_is_device_ptr(p)) return B200_OK;

  for (int q = 0; q < ss->n; ++q) {
    b200_stage_t *s = &ss->st[q];
    int same = views_same(s, p, rows, cols, rs, cs);
    int swapped = views_same(s, p, cols, rows, cs, rs);
    if (!same && !swapped) continue;
    /* The same host matrix staged again: if this use needs more of it than
     * the earlier one copied in, copy the whole view (and write back all of
     * it: the whole device copy is then valid). */
    const int want = !tri ? 0 : (same ? tri : (tri == 1 ? 2 : 1));
    if (s->tri && s->tri != want) {
      s->tri = 0;
      int st = stage_copy(s, ss->elt, 1);
      if (st != B200_OK) return st;
    }
    s->out |= out;
    /* Device strides of the staged copy in the requested orientation. */
    long drs = s->transposed ? s->ld : 1, dcs = s->transposed ? 1 : s->ld;
    v->ptr = s->dev;
    v->rs = same ? drs : dcs;
    v->cs = same ? dcs : drs;
    return B200_OK;
  }
  if (ss->n == (int)(sizeof ss->st / sizeof ss->st[0]))
    return b200_set_error(B200_EINVAL, "too many staged operands");

  b200_stage_t *s = &ss->st[ss->n];
  memset(s, 0, sizeof *s);
  s->host = p;
  s->rows = rows;
  s->cols = cols;
  s->rs = rs;
  s->cs = cs;
  s->out = out;
  s->tri = rows == cols ? tri : 0;
  s->transposed = rs != 1 && cs == 1;
  s->ld = s->transposed ? cols : rows;
  int st = b200_alloc(&s->dev, (size_t)rows * (size_t)cols * ss->elt);
  if (st != B200_OK) return st;
  ss->n++;
  if (copy_in) {
    st = stage_copy(s, ss->elt, 1);
    if (st != B200_OK) return st;
  }
  v->ptr = s->dev;
  v->rs = s->transposed ? s->ld : 1;
  v->cs = s->transposed ? 1 : s->ld;
  return B200_OK;
}

int b200_stage_end(b200_stage_set_t *ss, int status) {
  for (int q = 0; q < ss->n && status == B200_OK; ++q) {
    b200_stage_t *s = &ss->st[q];
    if (!s->out) continue;
    status = stage_copy(s, ss->elt, 0);
  }
  int sync = b200_stream_sync();
  for (int q = 0; q < ss->n; ++q) b200_free(ss->st[q].dev);
  ss->n = 0;
  if (status == B200_OK) status = sync;
  return status;
}

static size_t elt_of(int dtype) { return dtype == B200_F64 ? sizeof(double) : sizeof(float); }

/* A TRMM / TRSM panel is a whole triangular product or solve over the
 * panel's columns: below 2048 columns its inner products get too narrow to
 * fill the GPU (at n = 4096: 9.2 ms end to end for DTRSM with 1024-column
 * panels). */
enum { TRI_PANEL = 2048 };

/* Staged triangle of a SYMMETRIC / TRIANGULAR operand (1 lower, 2 upper), 0
 * for a general one. */
static int operand_tri(const mublis_l3_operand_t *o) {
  if (o->struc == MUBLIS_STRUC_GENERAL) return 0;
  return o->uplo == MUBLIS_LOWER ? 1 : o->uplo == MUBLIS_UPPER ? 2 : 0;
}

/* ---- column-panel pipelining of host operands ----------------------------
 *
 * A large call whose output columns are independent (no triangle restriction
 * on C, a plain op(B) whose columns feed only the same columns of C, or a
 * left TRSM / TRMM whose right-hand sides are independent) moves its output
 * and op(B) through the device in panels of columns, overlapping each
 * panel's transfers with the arithmetic of its neighbours
 * (b200_column_pipeline).  A is staged whole first. */

static int pipelinable(const void *p, long rows, long rs, long cs) {
  return p != NULL && !b200_is_device_ptr(p) && b200_colpipe_view_ok(rows, rs, cs);
}

static int l3_panel(void *ctx, long j0, long cols, void *in_dev, long in_rs, long in_cs,
                    void *out_dev, long out_rs, long out_cs) {
  (void)j0;
  b200_l3_desc_t d = *(const b200_l3_desc_t *)ctx;
  if (d.policy_n <= 0) d.policy_n = d.n;
  d.n = (int)cols;
  d.b[0] = in_dev ? in_dev : out_dev; /* in place when there is no separate input */
  d.rs_b[0] = in_dev ? in_rs : out_rs;
  d.cs_b[0] = in_dev ? in_cs : out_cs;
  d.c = out_dev;
  d.rs_c = out_rs;
  d.cs_c = out_cs;
  return b200_l3_run(&d);
}

/* Panel [j0, j0 + cols) of a lower-triangle output (SYRK / SYR2K): rows j0..
 * of C against rows j0.. of every A_t and columns j0.. of every B_t.  The
 * panel's C starts on the diagonal, so the ji relation is unchanged, and
 * each element is computed exactly as in the whole call. */
static int lower_panel(void *ctx, long j0, long cols, void *in_dev, long in_rs, long in_cs,
                       void *out_dev, long out_rs, long out_cs) {
  (void)in_dev, (void)in_rs, (void)in_cs;
  b200_l3_desc_t d = *(const b200_l3_desc_t *)ctx;
  const size_t elt = d.dtype == B200_F64 ? sizeof(double) : sizeof(float);
  if (d.policy_m <= 0) d.policy_m = d.m;
  if (d.policy_n <= 0) d.policy_n = d.n;
  for (int t = 0; t < d.npairs; ++t) {
    d.a[t] = (const char *)d.a[t] + j0 * d.rs_a[t] * (long)elt;
    d.b[t] = (const char *)d.b[t] + j0 * d.cs_b[t] * (long)elt;
  }
  d.m -= (int)j0;
  d.n = (int)cols;
  d.c = out_dev;
  d.rs_c = out_rs;
  d.cs_c = out_cs;
  return b200_l3_run(&d);
}

static int trsm_panel(void *ctx, long j0, long cols, void *in_dev, long in_rs, long in_cs,
                      void *out_dev, long out_rs, long out_cs) {
  (void)j0, (void)in_dev, (void)in_rs, (void)in_cs;
  b200_trsm_desc_t d = *(const b200_trsm_desc_t *)ctx;
  if (d.policy_n <= 0) d.policy_n = d.n;
  d.n = (int)cols;
  d.b = out_dev;
  d.rs_b = out_rs;
  d.cs_b = out_cs;
  return b200_trsm_run(&d);
}

/* Predicted time of the right-to-left lower-triangle pipeline with panel
 * widths w[0..np) (left to right) over an n x n lower C with k-deep
 * products: per panel, its blocks of the `nbuf` streamed operands and its
 * part of C cross PCIe one after another, its tiles run in rounds of
 * `slots` once those have arrived and the previous panel is done, and its
 * C goes back.  Seconds at 50 GB/s each way and `rate` flop/s. */
static double lower_plan_time(const long *w, int np, long n, long k, int npairs, int nbuf,
                              size_t elt, double rate, int slots) {
  const double bw = 50e9, tile = 128.0;
  const double round_s = 2.0 * tile * tile * (double)k * npairs / (rate / slots);
  double t_in = 0, t_comp = 0, t_out = 0;
  long j0 = n;
  for (int q = np - 1; q >= 0; --q) {
    j0 -= w[q];
    const double rows = (double)(n - j0), cols = (double)w[q];
    const double cbytes = (rows * cols - cols * cols / 2) * elt;
    t_in += (cbytes + cols * (double)k * elt * nbuf) / bw;
    const long tr = (n - j0 + 127) / 128, tc = (w[q] + 127) / 128;
    const long tiles = tc * tr - tc * (tc - 1) / 2; /* lower tiles of the panel */
    const long rounds = (tiles + slots - 1) / slots;
    t_comp = (t_in > t_comp ? t_in : t_comp) + rounds * round_s;
    t_out = (t_comp > t_out ? t_comp : t_out) + cbytes / bw;
  }
  return t_out;
}

/* Panel widths (multiples of n / 32, rounded to 128 columns) for the
 * right-to-left lower pipeline: the split into 2..4 panels with the least
 * predicted time.  The leftmost panel is the last one computed and copied
 * back, and the tallest, so the best splits keep it narrow (n = 4096 FP64
 * SYR2K: 512 | 640 | 896 | 2048).  Returns the panel count. */
static int lower_plan(long n, long k, int npairs, int nbuf, int dtype, long *w) {
  const size_t elt = elt_of(dtype);
  const double rate = dtype == B200_F64 ? 28e12 : 48e12;
  const int sms = b200_sm_count() > 0 ? b200_sm_count() : 148;
  const int slots = dtype == B200_F64 ? sms : 2 * sms;
  long u = (n / 32 + 127) / 128 * 128;
  if (u < 128) u = 128;
  const int units = (int)((n + u - 1) / u);
  double best = -1;
  int best_np = 0;
  long c[4];
  for (int a = 1; a < units; ++a)
    for (int b = a; b <= units; ++b)
      for (int e = b; e <= units; ++e) {
        /* cuts at a <= b <= e < units; equal cuts merge panels */
        const int cut[4] = {a, b, e, units};
        int np = 0;
        long prev = 0;
        for (int q = 0; q < 4; ++q) {
          const long x = cut[q] * u < n ? cut[q] * u : n;
          if (x > prev) c[np++] = x - prev, prev = x;
        }
        if (np < 2 || prev != n) continue;
        const double t = lower_plan_time(c, np, n, k, npairs, nbuf, elt, rate, slots);
        if (best < 0 || t < best) {
          best = t, best_np = np;
          for (int q = 0; q < np; ++q) w[q] = c[q];
        }
      }
  return best_np;
}

/* A one-pair product that writes only the lower triangle of a square C
 * (SYRK) as a pipeline over triangle panels of C: each column panel of C
 * below the diagonal is copied in, computed and copied back while its
 * neighbours move.  The panels run right to left, so the panel at column
 * j0 reads only rows j0.. of op(A) and columns j0.. of op(B): those
 * operands move in blocks beside the panels instead of before them
 * (streams), and the planner above picks the widths.  Two-pair products
 * (SYR2K) run this way only when every host operand can be streamed: with
 * the operands staged first, the pipeline lost to the whole call (DSYR2K
 * 4096^2: 12.4 -> 13.1 ms).  0 when the call does not qualify. */
static int try_pipeline_lower(const b200_l3_desc_t *d, int *status) {
  const mublis_l3_product_t *pr = &d->product;
  if (b200_serve_attached() || d->npairs < 1 || d->npairs > 2 || d->alpha == 0.0 || d->k <= 0 ||
      d->m != d->n || pr->domain.ji != MUBLIS_L3_LOWER || pr->domain.jp != MUBLIS_L3_ALL ||
      pr->domain.pi != MUBLIS_L3_ALL || pr->a.struc != MUBLIS_STRUC_GENERAL ||
      pr->b.struc != MUBLIS_STRUC_GENERAL || !pipelinable(d->c, d->m, d->rs_c, d->cs_c))
    return 0;
  /* Streaming needs a unit stride in every host operand. */
  int stream = 1;
  for (int t = 0; t < d->npairs; ++t) {
    if (d->a[t] == d->c || d->b[t] == d->c) return 0;
    if (!b200_is_device_ptr(d->a[t]) && d->rs_a[t] != 1 && d->cs_a[t] != 1) stream = 0;
    if (!b200_is_device_ptr(d->b[t]) && d->rs_b[t] != 1 && d->cs_b[t] != 1) stream = 0;
  }
  if (!stream && d->npairs != 1) return 0;
  const size_t elt = elt_of(d->dtype);
  if (b200_colpipe_panels(d->n, (size_t)d->m * d->n * elt / 2) < 2) return 0;
  b200_stage_set_t ss;
  b200_stage_begin(&ss, elt);
  b200_l3_desc_t dd = *d;
  b200_colpipe_t p;
  memset(&p, 0, sizeof p);
  b200_view_t v;
  int st = B200_OK;
  for (int t = 0; t < d->npairs && st == B200_OK; ++t)
    for (int side = 0; side < 2 && st == B200_OK; ++side) {
      const void *h = side ? d->b[t] : d->a[t];
      const long rs = side ? d->rs_b[t] : d->rs_a[t], cs = side ? d->cs_b[t] : d->cs_a[t];
      st = side ? b200_stage_view(&ss, h, d->k, d->n, rs, cs, !stream, 0, &v)
                : b200_stage_view(&ss, h, d->m, d->k, rs, cs, !stream, 0, &v);
      if (side)
        dd.b[t] = v.ptr, dd.rs_b[t] = v.rs, dd.cs_b[t] = v.cs;
      else
        dd.a[t] = v.ptr, dd.rs_a[t] = v.rs, dd.cs_a[t] = v.cs;
      if (st != B200_OK || !stream || v.ptr == h) continue; /* device-resident: not moved */
      int seen = 0;
      for (int q = 0; q < p.nstreams; ++q) seen |= p.streams[q].dev == v.ptr;
      if (seen) continue; /* another view of a matrix already moving */
      b200_colpipe_stream_t *s = &p.streams[p.nstreams++];
      s->host = h, s->rs = rs, s->cs = cs;
      s->dev = v.ptr, s->drs = v.rs, s->dcs = v.cs;
      s->extent = d->k;
      s->by_cols = side; /* rows j0.. of op(A), columns j0.. of op(B) */
    }
  if (st == B200_OK) {
    p.elt = elt;
    p.ncols = d->n;
    p.out.host = d->c, p.out.rows = d->m, p.out.rs = d->rs_c, p.out.cs = d->cs_c;
    p.out_read = 1; /* the diagonal blocks hold upper elements to return unchanged */
    p.out_lower = 1;
    p.run = lower_panel;
    p.ctx = &dd;
    if (stream) {
      p.reverse = 1;
      p.nwidths = lower_plan(d->n, d->k, d->npairs, p.nstreams, d->dtype, p.widths);
    }
    st = b200_column_pipeline(&p);
  }
  *status = b200_stage_end(&ss, st);
  return 1;
}

/* The l3 call as a pipeline over the columns of C, or 0 when it does not
 * qualify (the caller then stages everything at once). */
static int try_pipeline_l3(const b200_l3_desc_t *d, int *status) {
  if (b200_serve_attached() || d->npairs != 1 || d->alpha == 0.0 || d->k <= 0) return 0;
  const mublis_l3_product_t *pr = &d->product;
  if (pr->domain.ji != MUBLIS_L3_ALL || pr->domain.jp != MUBLIS_L3_ALL ||
      pr->b.struc != MUBLIS_STRUC_GENERAL || d->b[0] == d->c)
    return 0;
  if (!pipelinable(d->b[0], d->k, d->rs_b[0], d->cs_b[0]) ||
      !pipelinable(d->c, d->m, d->rs_c, d->cs_c))
    return 0;
  const size_t elt = elt_of(d->dtype);
  if (b200_colpipe_panels(d->n, (size_t)(d->k + d->m) * d->n * elt) < 2) return 0;
  b200_stage_set_t ss;
  b200_stage_begin(&ss, elt);
  b200_l3_desc_t dd = *d;
  b200_view_t v;
  int st = b200_stage_view_tri(&ss, d->a[0], d->m, d->k, d->rs_a[0], d->cs_a[0], 1, 0,
                               operand_tri(&pr->a), &v);
  dd.a[0] = v.ptr;
  dd.rs_a[0] = v.rs;
  dd.cs_a[0] = v.cs;
  if (st == B200_OK) {
    b200_colpipe_t p;
    memset(&p, 0, sizeof p);
    p.elt = elt;
    p.ncols = d->n;
    p.in.host = d->b[0], p.in.rows = d->k, p.in.rs = d->rs_b[0], p.in.cs = d->cs_b[0];
    p.out.host = d->c, p.out.rows = d->m, p.out.rs = d->rs_c, p.out.cs = d->cs_c;
    p.out_read = d->beta != 0.0;
    p.run = l3_panel;
    p.ctx = &dd;
    st = b200_column_pipeline(&p);
  }
  *status = b200_stage_end(&ss, st);
  return 1;
}

int b200_front_l3(b200_l3_desc_t *d) {
  if (d->m == 0 || d->n == 0) return B200_OK;
  if (d->m < 0 || d->n < 0 || d->k < 0) return b200_set_error(B200_EINVAL, "negative size");
  int st = b200_init();
  if (st != B200_OK) return st;
  if (try_pipeline_l3(d, &st)) return st;
  if (try_pipeline_lower(d, &st)) return st;

  b200_stage_set_t ss;
  b200_stage_begin(&ss, elt_of(d->dtype));
  b200_l3_desc_t dd = *d;
  const int update = d->alpha != 0.0 && d->k > 0;
  b200_view_t v;
  /* A symmetric or triangular operand is read in its stored triangle only,
   * and a ji-restricted C is read (beta != 0) and written in its triangle
   * only: just those triangles cross PCIe. */
  const mublis_l3_product_t *pr = &d->product;
  const int a_tri = operand_tri(&pr->a), b_tri = operand_tri(&pr->b);
  const int c_tri = pr->domain.ji == MUBLIS_L3_LOWER ? 1 : pr->domain.ji == MUBLIS_L3_UPPER ? 2 : 0;
  for (int t = 0; t < d->npairs && update && st == B200_OK; ++t) {
    st = b200_stage_view_tri(&ss, d->a[t], d->m, d->k, d->rs_a[t], d->cs_a[t], 1, 0, a_tri, &v);
    dd.a[t] = v.ptr;
    dd.rs_a[t] = v.rs;
    dd.cs_a[t] = v.cs;
    if (st != B200_OK) break;
    st = b200_stage_view_tri(&ss, d->b[t], d->k, d->n, d->rs_b[t], d->cs_b[t], 1, 0, b_tri, &v);
    dd.b[t] = v.ptr;
    dd.rs_b[t] = v.rs;
    dd.cs_b[t] = v.cs;
  }
  if (st == B200_OK) {
    /* A triangle-staged C is copied in even when beta == 0: the column
     * blocks that straddle the diagonal also hold elements of the other
     * triangle, which the write-back must return unchanged. */
    st = b200_stage_view_tri(&ss, d->c, d->m, d->n, d->rs_c, d->cs_c,
                             d->beta != 0.0 || c_tri != 0, 1, c_tri, &v);
    dd.c = v.ptr;
    dd.rs_c = v.rs;
    dd.cs_c = v.cs;
  }
  /* Device-resident calls go through the request server when one is
   * attached (continuous batching across calling threads). */
  if (st == B200_OK) st = ss.n == 0 && b200_serve_attached() ? b200_serve_l3(&dd) : b200_l3_run(&dd);
  return b200_stage_end(&ss, st);
}

static mublis_uplo_t flip(mublis_uplo_t u) {
  return u == MUBLIS_LOWER ? MUBLIS_UPPER : (u == MUBLIS_UPPER ? MUBLIS_LOWER : MUBLIS_DENSE);
}

int b200_front_trmm(int dtype, mublis_side_t side, mublis_uplo_t uplo, mublis_trans_t trans,
                    mublis_diag_t diag, int m, int n, double alpha, const void *a, int rs_a,
                    int cs_a, void *b, int rs_b, int cs_b) {
  if (m == 0 || n == 0) return B200_OK;
  if (m < 0 || n < 0) return b200_set_error(B200_EINVAL, "negative size");
  int st = b200_init();
  if (st != B200_OK) return st;
  b200_stage_set_t ss;
  b200_stage_begin(&ss, elt_of(dtype));
  b200_view_t vb, va;
  /* Left side with host B: the right-hand sides are independent, so B goes
   * through the device in column panels (B stays unstaged here). */
  const int piped = side == MUBLIS_LEFT && alpha != 0.0 && !b200_serve_attached() &&
                    pipelinable(b, m, rs_b, cs_b) &&
                    b200_colpipe_panels_min(n, (size_t)m * n * elt_of(dtype), TRI_PANEL) >= 2;
  if (piped) {
    vb.ptr = b, vb.rs = rs_b, vb.cs = cs_b;
  } else {
    st = b200_stage_view(&ss, b, m, n, rs_b, cs_b, alpha != 0.0, 1, &vb);
  }
  if (st == B200_OK && alpha == 0.0) {
    st = b200_scale_strided(dtype, m, n, 0.0, vb.ptr, vb.rs, vb.cs, MUBLIS_L3_ALL);
    return b200_stage_end(&ss, st);
  }
  int ka = side == MUBLIS_LEFT ? m : n;
  /* Only the stored triangle of A is read: only it crosses PCIe. */
  if (st == B200_OK)
    st = b200_stage_view_tri(&ss, a, ka, ka, rs_a, cs_a, 1, 0, uplo == MUBLIS_UPPER ? 2 : 1, &va);
  if (st != B200_OK) return b200_stage_end(&ss, st);

  long ars = va.rs, acs = va.cs;
  if (trans == MUBLIS_TRANSPOSE) { /* trmm.c:44-49 */
    long t = ars; ars = acs; acs = t;
    uplo = flip(uplo);
  }
  mublis_l3_relation_t tri = uplo == MUBLIS_LOWER ? MUBLIS_L3_LOWER : MUBLIS_L3_UPPER;
  mublis_l3_operand_t gen = {MUBLIS_STRUC_GENERAL, MUBLIS_DENSE, MUBLIS_PACKM_DIAG_NONUNIT};
  mublis_l3_operand_t trio = {MUBLIS_STRUC_TRIANGULAR, uplo,
                              diag == MUBLIS_UNIT_DIAG ? MUBLIS_PACKM_DIAG_UNIT
                                                       : MUBLIS_PACKM_DIAG_NONUNIT};
  b200_l3_desc_t d;
  memset(&d, 0, sizeof d);
  d.dtype = dtype;
  d.m = m;
  d.n = n;
  d.alpha = alpha;
  d.beta = 0.0;
  d.npairs = 1;
  d.form = B200_FORM_AUTO;
  d.product.domain.ji = MUBLIS_L3_ALL;
  if (side == MUBLIS_LEFT) { /* trmm.c:51-82,98-106 */
    d.k = m;
    d.product.domain.pi = tri;
    d.product.domain.jp = MUBLIS_L3_ALL;
    d.product.a = trio;
    d.product.b = gen;
    d.a[0] = va.ptr; d.rs_a[0] = ars; d.cs_a[0] = acs;
    d.b[0] = vb.ptr; d.rs_b[0] = vb.rs; d.cs_b[0] = vb.cs;
  } else {
    d.k = n;
    d.product.domain.jp = tri;
    d.product.domain.pi = MUBLIS_L3_ALL;
    d.product.a = gen;
    d.product.b = trio;
    d.a[0] = vb.ptr; d.rs_a[0] = vb.rs; d.cs_a[0] = vb.cs;
    d.b[0] = va.ptr; d.rs_b[0] = ars; d.cs_b[0] = acs;
  }
  /* In place: the device driver packs both operands before the contraction
   * writes C, so C may alias B. */
  d.c = vb.ptr;
  d.rs_c = vb.rs;
  d.cs_c = vb.cs;
  if (piped) {
    b200_colpipe_t p;
    memset(&p, 0, sizeof p);
    p.elt = elt_of(dtype);
    p.ncols = n;
    p.out.host = b, p.out.rows = m, p.out.rs = rs_b, p.out.cs = cs_b;
    p.out_read = 1;
    p.run = l3_panel;
    p.ctx = &d;
    p.panel_min = TRI_PANEL;
    st = b200_column_pipeline(&p);
    return b200_stage_end(&ss, st);
  }
  st = ss.n == 0 && b200_serve_attached() ? b200_serve_l3(&d) : b200_l3_run(&d);
  return b200_stage_end(&ss, st);
}

int b200_front_trsm(int dtype, mublis_side_t side, mublis_uplo_t uplo, mublis_trans_t trans,
                    mublis_diag_t diag, int m, int n, double alpha, const void *a, int rs_a,
                    int cs_a, void *b, int rs_b, int cs_b) {
  if (m == 0 || n == 0) return B200_OK;
  if (m < 0 || n < 0) return b200_set_error(B200_EINVAL, "negative size");
  int st = b200_init();
  if (st != B200_OK) return st;
  b200_stage_set_t ss;
  b200_stage_begin(&ss, elt_of(dtype));
  b200_view_t vb, va;
  /* Host B: the right-hand sides (columns of the normalised left solve) are
   * independent, so B goes through the device in panels (unstaged here). */
  const long m_left = side == MUBLIS_LEFT ? m : n, n_left = side == MUBLIS_LEFT ? n : m;
  const long rs_left = side == MUBLIS_LEFT ? rs_b : cs_b, cs_left = side == MUBLIS_LEFT ? cs_b : rs_b;
  const int piped = alpha != 0.0 && !b200_serve_attached() &&
                    pipelinable(b, m_left, rs_left, cs_left) &&
                    b200_colpipe_panels_min(n_left, (size_t)m * n * elt_of(dtype), TRI_PANEL) >= 2;
  if (piped) {
    vb.ptr = b, vb.rs = rs_b, vb.cs = cs_b;
  } else {
    st = b200_stage_view(&ss, b, m, n, rs_b, cs_b, alpha != 0.0, 1, &vb);
  }
  if (st == B200_OK && alpha == 0.0) { /* trsm.c:27-33 */
    st = b200_scale_strided(dtype, m, n, 0.0, vb.ptr, vb.rs, vb.cs, MUBLIS_L3_ALL);
    return b200_stage_end(&ss, st);
  }
  int ka = side == MUBLIS_LEFT ? m : n;
  /* Only the stored triangle of A is read: only it crosses PCIe. */
  if (st == B200_OK)
    st = b200_stage_view_tri(&ss, a, ka, ka, rs_a, cs_a, 1, 0, uplo == MUBLIS_UPPER ? 2 : 1, &va);
  if (st != B200_OK) return b200_stage_end(&ss, st);

  long brs = vb.rs, bcs = vb.cs, ars = va.rs, acs = va.cs;
  if (side == MUBLIS_RIGHT) { /* trsm.c:35-47 */
    int t = m; m = n; n = t;
    long u = brs; brs = bcs; bcs = u;
    trans = trans == MUBLIS_NO_TRANSPOSE ? MUBLIS_TRANSPOSE : MUBLIS_NO_TRANSPOSE;
  }
  if (trans == MUBLIS_TRANSPOSE) { /* trsm.c:49-54 */
    long u = ars; ars = acs; acs = u;
    uplo = flip(uplo);
  }
  b200_trsm_desc_t d;
  memset(&d, 0, sizeof d);
  d.dtype = dtype;
  d.m = m;
  d.n = n;
  d.alpha = alpha;
  d.a = va.ptr;
  d.rs_a = ars;
  d.cs_a = acs;
  d.b = vb.ptr;
  d.rs_b = brs;
  d.cs_b = bcs;
  d.uplo = uplo;
  d.unit_diag = diag == MUBLIS_UNIT_DIAG;
  d.form = B200_FORM_AUTO;
  if (piped) {
    b200_colpipe_t p;
    memset(&p, 0, sizeof p);
    p.elt = elt_of(dtype);
    p.ncols = n;
    p.out.host = b, p.out.rows = m, p.out.rs = brs, p.out.cs = bcs;
    p.out_read = 1;
    p.run = trsm_panel;
    p.ctx = &d;
    p.panel_min = TRI_PANEL;
    /* The diagonal inverses depend on A only: built once for all panels. */
    void *prep = NULL;
    d.policy_n = n;
    st = b200_trsm_prepare(&d, &prep);
    d.prep = prep;
    if (st == B200_OK) st = b200_column_pipeline(&p);
    b200_trsm_release(prep);
    return b200_stage_end(&ss, st);
  }
  st = ss.n == 0 && b200_serve_attached() ? b200_serve_trsm(&d) : b200_trsm_run(&d);
  return b200_stage_end(&ss, st);
}

/* ---- mublis_l3_{s,d}driver ---------------------------------------------- */

static int driver(int dtype, int m, int n, int k, double alpha, const void *a, int rs_a,
                  int cs_a, const void *b, int rs_b, int cs_b, double beta, void *c, int rs_c,
                  int cs_c, const mublis_l3_product_t *product) {
  if (m == 0 || n == 0) return 0;
  if (product == NULL) return b200_set_error(B200_EINVAL, "null product descriptor");
  b200_l3_desc_t d;
  memset(&d, 0, sizeof d);
  d.dtype = dtype;
  d.m = m;
  d.n = n;
  d.k = k;
  d.alpha = alpha;
  d.beta = beta;
  d.npairs = 1;
  d.a[0] = a; d.rs_a[0] = rs_a; d.cs_a[0] = cs_a;
  d.b[0] = b; d.rs_b[0] = rs_b; d.cs_b[0] = cs_b;
  d.c = c; d.rs_c = rs_c; d.cs_c = cs_c;
  d.product = *product;
  d.form = B200_FORM_AUTO;
  return b200_front_l3(&d);
}

int mublis_l3_sdriver(int m, int n, int k, float alpha, const float *a, int rs_a, int cs_a,
                      const float *b, int rs_b, int cs_b, float beta, float *c, int rs_c,
                      int cs_c, const mublis_l3_product_t *product) {
  return driver(B200_F32, m, n, k, alpha, a, rs_a, cs_a, b, rs_b, cs_b, beta, c, rs_c, cs_c,
                product);
}

int mublis_l3_ddriver(int m, int n, int k, double alpha, const double *a, int rs_a, int cs_a,
                      const double *b, int rs_b, int cs_b, double beta, double *c, int rs_c,
                      int cs_c, const mublis_l3_product_t *product) {
  return driver(B200_F64, m, n, k, alpha, a, rs_a, cs_a, b, rs_b, cs_b, beta, c, rs_c, cs_c,
                product);
}
