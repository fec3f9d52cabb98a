// runtime.cu -- device bring-up, per-thread streams, stream-ordered scratch,
// strided host<->device staging, error strings, default precision forms and
// the per-kernel event profiler of libmublis.
//
// The reference has no device; its runtime pieces are the pthread_once
// context (frame/base/safe_dispatch.c:6,64) and the mutex-guarded block pool
// (frame/base/pool.c:23-66,233-318).  Here the once-init brings up the CUDA
// device, and the pool is CUDA's stream-ordered allocator (cudaMallocAsync on
// the calling thread's stream, with the pool's release threshold raised so
// freed blocks stay cached for the next call).
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "../../include/mublis_b200.h"

namespace {

std::once_flag g_init_once;
int g_init_status = B200_ECUDA;
int g_device = 0;
std::atomic<unsigned long long> g_launches{0};

int g_default_form[2] = {B200_FORM_PLAIN, B200_FORM_PLAIN};
int g_default_slices[2] = {0, 0};  // per dtype: slice / modulus count, 0 = form default
double g_default_target[2] = {0.0, 0.0};  // per dtype: "ozaki2@<target>" error target, 0 = none

thread_local cudaStream_t t_stream = nullptr;
thread_local bool t_stream_owned = false;
thread_local char t_error[512] = "";

struct ProfRec {
  const char *name;
  cudaEvent_t start, stop;
};
std::mutex g_prof_mu;
std::vector<ProfRec> g_prof;
std::atomic<int> g_prof_on{0};

void do_init() {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    snprintf(t_error, sizeof t_error, "no CUDA device: %s",
             e == cudaSuccess ? "device count is 0" : cudaGetErrorString(e));
    g_init_status = B200_ECUDA;
    return;
  }
  cudaGetDevice(&g_device);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, g_device) != cudaSuccess || prop.major != 10) {
    snprintf(t_error, sizeof t_error,
             "libmublis is built for sm_100a (B200); device %d is sm_%d%d", g_device,
             prop.major, prop.minor);
    g_init_status = B200_ECUDA;
    return;
  }
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, g_device) == cudaSuccess) {
    uint64_t threshold = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  int slices = 0;
  int sslices = 0;
  double starget = 0.0, dtarget = 0.0;
  int sf = b200_parse_form(getenv("MUBLIS_B200_SFORM"), &sslices, &starget);
  int df = b200_parse_form(getenv("MUBLIS_B200_DFORM"), &slices, &dtarget);
  if (sf == B200_FORM_PLAIN || sf == B200_FORM_BF16X3 || sf == B200_FORM_BF16X6 ||
      sf == B200_FORM_FP16X3 || sf == B200_FORM_OZAKI2 || sf == B200_FORM_POLICY)
    g_default_form[B200_F32] = sf;
  if (df == B200_FORM_PLAIN || df == B200_FORM_OZAKI || df == B200_FORM_OZAKI2 ||
      df == B200_FORM_POLICY)
    g_default_form[B200_F64] = df;
  if (slices > 0) g_default_slices[B200_F64] = slices;
  if (sslices > 0) g_default_slices[B200_F32] = sslices;
  if (df == B200_FORM_OZAKI2) g_default_target[B200_F64] = dtarget;
  if (sf == B200_FORM_OZAKI2) g_default_target[B200_F32] = starget;
  g_init_status = B200_OK;
  b200_tune_autoload();
  // The allocation-free SGEMM's fixed scratch array is claimed here, at
  // start-up, rather than on that entry point's first call.
  b200_noalloc_setup();
}

}  // namespace

void b200_note_cuda_error(cudaError_t err, const char *what, const char *file, int line) {
  snprintf(t_error, sizeof t_error, "%s:%d: %s -> %s", file, line, what,
           cudaGetErrorString(err));
  if (getenv("MUBLIS_B200_VERBOSE")) fprintf(stderr, "libmublis: %s\n", t_error);
}

B200ProfScope::B200ProfScope(const char *name, cudaStream_t s) : slot(-1), stream(s) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (!g_prof_on.load(std::memory_order_relaxed)) return;
  ProfRec r{name, nullptr, nullptr};
  cudaEventCreate(&r.start);
  cudaEventCreate(&r.stop);
  cudaEventRecord(r.start, s);
  std::lock_guard<std::mutex> lk(g_prof_mu);
  slot = (int)g_prof.size();
  g_prof.push_back(r);
}

B200ProfScope::~B200ProfScope() {
  if (slot < 0) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  cudaEventRecord(g_prof[slot].stop, stream);
}

extern "C" {

int b200_init(void) {
  std::call_once(g_init_once, do_init);
  if (g_init_status != B200_OK && !t_error[0])
    snprintf(t_error, sizeof t_error, "CUDA device unavailable");
  return g_init_status;
}

int b200_device_count(void) {
  int c = 0;
  return cudaGetDeviceCount(&c) == cudaSuccess ? c : 0;
}

int b200_is_device_ptr(const void *p) {
  if (!p) return 0;
  cudaPointerAttributes attr;
  cudaError_t e = cudaPointerGetAttributes(&attr, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

// A stream that library code switches to for part of one call (the
// second column half of a large triangular solve); the thread's own stream
// and its ownership are untouched.
thread_local cudaStream_t t_override = nullptr;
// Second streams, one per stream this thread issues on (a request server's
// scheduler thread issues on several), so that concurrent calls on
// different streams do not queue behind each other on a shared one.
constexpr int AUX_SLOTS = 8;
thread_local cudaStream_t t_aux_of[AUX_SLOTS] = {}, t_aux[AUX_SLOTS] = {};

void *b200_override_stream(void *stream) {
  void *prev = (void *)t_override;
  t_override = (cudaStream_t)stream;
  return prev;
}

void *b200_aux_stream(void) {
  const cudaStream_t cur = (cudaStream_t)b200_stream();
  int slot = -1;
  for (int i = 0; i < AUX_SLOTS; ++i) {
    if (t_aux[i] && t_aux_of[i] == cur) return (void *)t_aux[i];
    if (!t_aux[i] && slot < 0) slot = i;
  }
  if (slot < 0) return nullptr;  // more primary streams than slots: no second stream
  if (cudaStreamCreateWithFlags(&t_aux[slot], cudaStreamNonBlocking) != cudaSuccess) {
    t_aux[slot] = nullptr;
    return nullptr;
  }
  t_aux_of[slot] = cur;
  return (void *)t_aux[slot];
}

void *b200_stream(void) {
  if (t_override) return (void *)t_override;
  if (!t_stream) {
    cudaStreamCreateWithFlags(&t_stream, cudaStreamNonBlocking);
    t_stream_owned = true;
  }
  return (void *)t_stream;
}

int b200_set_thread_stream(void *stream) {
  if (t_stream && t_stream_owned) cudaStreamDestroy(t_stream);
  t_stream = (cudaStream_t)stream;
  t_stream_owned = false;
  return B200_OK;
}

int b200_stream_sync(void) {
  B200_CUDA_TRY(cudaStreamSynchronize(b200_cur_stream()));
  if (int e = b200_take_device_error())
    return b200_set_error(e, "a device-side bounded wait timed out (kernel aborted)");
  return B200_OK;
}

int b200_alloc(void **p, size_t bytes) {
  *p = nullptr;
  if (bytes == 0) bytes = 256;
  B200_CUDA_TRY(cudaMallocAsync(p, bytes, b200_cur_stream()));
  return B200_OK;
}

void b200_free(void *p) {
  if (p) cudaFreeAsync(p, b200_cur_stream());
}

namespace {
std::atomic<unsigned long long> g_test_stall{0};
constexpr unsigned long long B200_TEST_STALL_MAX_NS = 2000000000ull;
}  // namespace

int mublis_b200_test_stall_next(unsigned long long wait_limit_ns) {
  if (wait_limit_ns == 0 || wait_limit_ns > B200_TEST_STALL_MAX_NS)
    return b200_set_error(B200_EINVAL, "test_stall_next: limit must be in (0, 2 s]");
  g_test_stall.store(wait_limit_ns);
  return B200_OK;
}

unsigned long long b200_take_test_stall(void) { return g_test_stall.exchange(0); }

int b200_set_error(int code, const char *where) {
  snprintf(t_error, sizeof t_error, "%s", where);
  return code;
}

const char *b200_last_error(void) { return t_error; }

int b200_sm_count(void) {
  static std::atomic<int> cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  int sms = cache[dev].load(std::memory_order_relaxed);
  if (!sms) {
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
      sms = 148;
    cache[dev].store(sms, std::memory_order_relaxed);
  }
  return sms;
}

int b200_parse_form(const char *s, int *slices, double *target) {
  if (!s || !*s) return B200_FORM_AUTO;
  if (!strcmp(s, "plain")) return B200_FORM_PLAIN;
  if (!strcmp(s, "bf16x3")) return B200_FORM_BF16X3;
  if (!strcmp(s, "bf16x6")) return B200_FORM_BF16X6;
  if (!strcmp(s, "fp16x3")) return B200_FORM_FP16X3;
  if (!strcmp(s, "auto")) return B200_FORM_POLICY;
  const bool mod = !strncmp(s, "ozaki2", 6);
  if (mod || !strncmp(s, "ozaki", 5)) {
    const char *tail = s + (mod ? 6 : 5);
    if (*tail == ':') {
      if (slices) *slices = atoi(tail + 1);
    } else if (mod && *tail == '@') {
      char *end = nullptr;
      const double t = strtod(tail + 1, &end);
      if (!(t > 0) || end == tail + 1 || *end) return B200_FORM_AUTO;
      if (target) *target = t;
    } else if (*tail) {
      return B200_FORM_AUTO;
    }
    return mod ? B200_FORM_OZAKI2 : B200_FORM_OZAKI;
  }
  return B200_FORM_AUTO;
}

int b200_get_default_form(int dtype) { return g_default_form[dtype == B200_F64]; }
double b200_get_default_target(int dtype) { return g_default_target[dtype == B200_F64]; }
int b200_get_default_slices(int dtype) { return g_default_slices[dtype == B200_F64]; }

int b200_set_default_form(int dtype, int form, int slices) {
  if (dtype == B200_F32 && form != B200_FORM_PLAIN && form != B200_FORM_BF16X3 &&
      form != B200_FORM_BF16X6 && form != B200_FORM_FP16X3 && form != B200_FORM_OZAKI2 &&
      form != B200_FORM_POLICY)
    return B200_EINVAL;
  if (dtype == B200_F64 && form != B200_FORM_PLAIN && form != B200_FORM_OZAKI &&
      form != B200_FORM_OZAKI2 && form != B200_FORM_POLICY)
    return B200_EINVAL;
  g_default_form[dtype == B200_F64] = form;
  // The count and target belong to the form just set (0: that form's own
  // default).
  g_default_slices[dtype == B200_F64] = slices > 0 ? slices : 0;
  g_default_target[dtype == B200_F64] = 0.0;
  return B200_OK;
}

// Host -> compact device (column-major rows x cols, leading dimension ld).
namespace {

// Helper streams for host-to-device copies, one per stream that issues them
// on this thread, with the fork / join events of the split.
constexpr int COPY_SLOTS = 4;
struct CopyHelper {
  cudaStream_t of = nullptr, helper = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
thread_local CopyHelper t_copy_helpers[COPY_SLOTS];

CopyHelper *copy_helper(cudaStream_t s) {
  for (auto &c : t_copy_helpers)
    if (c.helper && c.of == s) return &c;
  for (auto &c : t_copy_helpers) {
    if (c.helper) continue;
    if (cudaStreamCreateWithFlags(&c.helper, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c.join, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    c.of = s;
    return &c;
  }
  return nullptr;
}

}  // namespace

// Host-to-device 2-D copy (height rows of width bytes).  A large one is cut
// in two halves, issued on s and on a helper stream paired with s (forked
// from and joined back into s), so that two copy engines share the link:
// one host-to-device copy moved 43 GB/s over this B200's PCIe Gen5 x16
// link, two at once 55 GB/s (device-to-host: 56 either way).
cudaError_t b200_h2d_2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
                        size_t height, cudaStream_t s) {
  CopyHelper *h = width * height >= ((size_t)8 << 20) && height >= 2 ? copy_helper(s) : nullptr;
  if (!h) return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyHostToDevice, s);
  const size_t h1 = height / 2;
  cudaError_t e = cudaEventRecord(h->fork, s);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(h->helper, h->fork, 0);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, h1, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpy2DAsync((char *)dst + h1 * dpitch, dpitch, (const char *)src + h1 * spitch,
                          spitch, width, height - h1, cudaMemcpyHostToDevice, h->helper);
  if (e == cudaSuccess) e = cudaEventRecord(h->join, h->helper);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s, h->join, 0);
  return e;
}

int b200_copy_h2d(void *dst, long ld, const void *src, long rs, long cs, long rows, long cols,
                  size_t elt) {
  if (rows <= 0 || cols <= 0) return B200_OK;
  cudaStream_t s = b200_cur_stream();
  if (rs == 1 && (cols == 1 || cs >= rows)) {
    B200_CUDA_TRY(b200_h2d_2d(dst, ld * elt, src, (cols == 1 ? rows : cs) * elt, rows * elt, cols,
                              s));
    return B200_OK;
  }
  // General strides: gather on the host into a contiguous staging block.
  size_t bytes = (size_t)rows * cols * elt;
  char *stage = (char *)malloc(bytes);
  if (!stage) return b200_set_error(B200_ENOMEM, "host staging allocation failed");
  const char *s8 = (const char *)src;
  for (long j = 0; j < cols; ++j)
    for (long i = 0; i < rows; ++i)
      memcpy(stage + (i + j * rows) * elt, s8 + (i * rs + j * cs) * (long)elt, elt);
  cudaError_t e = cudaMemcpy2DAsync(dst, ld * elt, stage, rows * elt, rows * elt, cols,
                                    cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  free(stage);
  B200_CUDA_TRY(e);
  return B200_OK;
}

int b200_copy_d2h(void *dst, long rs, long cs, const void *src, long ld, long rows, long cols,
                  size_t elt) {
  if (rows <= 0 || cols <= 0) return B200_OK;
  cudaStream_t s = b200_cur_stream();
  if (rs == 1 && (cols == 1 || cs >= rows)) {
    B200_CUDA_TRY(cudaMemcpy2DAsync(dst, (cols == 1 ? rows : cs) * elt, src, ld * elt,
                                    rows * elt, cols, cudaMemcpyDeviceToHost, s));
    return B200_OK;
  }
  size_t bytes = (size_t)rows * cols * elt;
  char *stage = (char *)malloc(bytes);
  if (!stage) return b200_set_error(B200_ENOMEM, "host staging allocation failed");
  cudaError_t e = cudaMemcpy2DAsync(stage, rows * elt, src, ld * elt, rows * elt, cols,
                                    cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) {
    char *d8 = (char *)dst;
    for (long j = 0; j < cols; ++j)
      for (long i = 0; i < rows; ++i)
        memcpy(d8 + (i * rs + j * cs) * (long)elt, stage + (i + j * rows) * elt, elt);
  }
  free(stage);
  B200_CUDA_TRY(e);
  return B200_OK;
}

// ---- column-panel pipeline (host-resident operands) --------------------------

namespace {

thread_local cudaStream_t t_copy_in = nullptr, t_copy_out = nullptr;

int copy_streams() {
  if (!t_copy_in) B200_CUDA_TRY(cudaStreamCreateWithFlags(&t_copy_in, cudaStreamNonBlocking));
  if (!t_copy_out) B200_CUDA_TRY(cudaStreamCreateWithFlags(&t_copy_out, cudaStreamNonBlocking));
  return B200_OK;
}

// Panel [j0, j0 + cols) of a host view as a 2-D copy.  rs == 1: columns are
// contiguous, the device panel is column-major (ld = rows).  cs == 1: rows
// are contiguous, the device panel is row-major (ld = cols).
struct PanelCopy {
  size_t width, height, hpitch, dpitch;
  long off, drs, dcs;
};

// Rows [r0, v.rows) of panel [j0, j0 + cols) of a host view.
PanelCopy panel_copy(const b200_colpipe_view_t &v, long j0, long cols, size_t elt, long r0 = 0) {
  PanelCopy c;
  const long rows = v.rows - r0;
  if (v.rs == 1) {
    c.width = rows * elt, c.height = cols, c.hpitch = (cols == 1 ? v.rows : v.cs) * elt;
    c.dpitch = rows * elt, c.off = j0 * v.cs + r0, c.drs = 1, c.dcs = rows;
  } else {
    c.width = cols * elt, c.height = rows, c.hpitch = v.rs * elt;
    c.dpitch = cols * elt, c.off = r0 * v.rs + j0, c.drs = cols, c.dcs = 1;
  }
  return c;
}

// A lower-triangle output panel [j0, j0 + cols) (device panel from element
// (j0, j0), strides co.drs / co.dcs) moved in blocks of 128 columns, each
// from its first column's diagonal down, so the part of the panel's
// diagonal block above the diagonal crosses PCIe only within 128 x 128
// squares.
cudaError_t lower_panel_copy(const b200_colpipe_view_t &v, long j0, long cols, size_t elt,
                             void *dev, const PanelCopy &co, bool to_device, cudaStream_t s) {
  constexpr long SUB = 128;
  for (long c0 = j0; c0 < j0 + cols; c0 += SUB) {
    const long nc = j0 + cols - c0 < SUB ? j0 + cols - c0 : SUB, nr = v.rows - c0;
    if (nr <= 0) break;
    char *d = (char *)dev + ((c0 - j0) * co.drs + (c0 - j0) * co.dcs) * (long)elt;
    char *h = (char *)v.host + (c0 * v.rs + c0 * v.cs) * (long)elt;
    const bool colmajor = v.rs == 1;
    const size_t width = (colmajor ? nr : nc) * elt, height = colmajor ? nc : nr;
    const size_t hpitch = (colmajor ? v.cs : v.rs) * elt;
    const size_t dpitch = (colmajor ? co.dcs : co.drs) * elt;
    const cudaError_t e =
        to_device ? b200_h2d_2d(d, dpitch, h, hpitch, width, height, s)
                  : cudaMemcpy2DAsync(h, hpitch, d, dpitch, width, height, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace

int b200_colpipe_view_ok(long rows, long rs, long cs) {
  return rs == 1 ? cs >= rows : (cs == 1 && rs >= 1);
}

int b200_colpipe_panels_min(long ncols, size_t bytes, long min_cols) {
  if (bytes < (32u << 20) || min_cols <= 0) return 1;
  long p = ncols / min_cols;
  return (int)(p > 4 ? 4 : p);
}

int b200_colpipe_panels(long ncols, size_t bytes) {
  return b200_colpipe_panels_min(ncols, bytes, 1024);
}

int b200_column_pipeline(const b200_colpipe_t *p) {
  B200_TRY(copy_streams());
  cudaStream_t sc = b200_cur_stream(), si = t_copy_in, so = t_copy_out;
  // Panels [start[q], start[q] + width[q]), left to right.
  long width[B200_COLPIPE_MAX_PANELS], start[B200_COLPIPE_MAX_PANELS];
  int np = 0;
  if (p->nwidths > 0) {
    if (p->nwidths > B200_COLPIPE_MAX_PANELS)
      return b200_set_error(B200_EINVAL, "pipeline: too many panels");
    long sum = 0;
    for (int q = 0; q < p->nwidths; ++q) {
      if (p->widths[q] <= 0) return b200_set_error(B200_EINVAL, "pipeline: empty panel");
      start[q] = sum, width[q] = p->widths[q], sum += p->widths[q];
    }
    if (sum != p->ncols) return b200_set_error(B200_EINVAL, "pipeline: panels do not cover C");
    np = p->nwidths;
  } else {
    const int npan =
        b200_colpipe_panels_min(p->ncols, 1ull << 40, p->panel_min > 0 ? p->panel_min : 1024);
    const long w0 = b200_round_up(b200_ceil_div(p->ncols, npan < 1 ? 1 : npan), 128);
    // Half-width first and last panels: the first computation starts after
    // a smaller copy-in, and the last one (and its copy back, which nothing
    // overlaps) is shorter.  MUBLIS_B200_PIPE_EDGES=0 keeps even panels.
    static const bool edges = [] {
      const char *e = getenv("MUBLIS_B200_PIPE_EDGES");
      return !(e && !strcmp(e, "0"));
    }();
    const long half = b200_round_up(w0 / 2, 128);
    // (Calls whose panels must stay wide -- TRSM / TRMM, panel_min 2048 --
    // keep even panels.)
    if (edges && p->panel_min <= 1024 && npan >= 2 && half < w0 &&
        npan + 1 <= B200_COLPIPE_MAX_PANELS && (p->ncols - half) / 128 * 128 > half) {
      start[0] = 0, width[0] = half, np = 1;
      // The last panel starts on a multiple of 128, like every other one.
      const long last = (p->ncols - half) / 128 * 128;
      for (long j0 = half; j0 < last && np < B200_COLPIPE_MAX_PANELS - 1; ++np) {
        const long wq = last - j0 < w0 ? last - j0 : w0;
        start[np] = j0, width[np] = wq, j0 += wq;
      }
      start[np] = last, width[np] = p->ncols - last, ++np;
    } else {
      for (long j0 = 0; j0 < p->ncols && np < B200_COLPIPE_MAX_PANELS; j0 += w0, ++np)
        start[np] = j0, width[np] = p->ncols - j0 < w0 ? p->ncols - j0 : w0;
    }
  }
  if (p->nstreams < 0 || p->nstreams > B200_COLPIPE_MAX_STREAMS)
    return b200_set_error(B200_EINVAL, "pipeline: too many streamed operands");
  for (int t = 0; t < p->nstreams; ++t) {
    const b200_colpipe_stream_t &s = p->streams[t];
    if (!((s.rs == 1 && s.drs == 1) || (s.cs == 1 && s.dcs == 1)))
      return b200_set_error(B200_EINVAL, "pipeline: streamed operand has no unit stride");
  }
  long w = 0;
  for (int q = 0; q < np; ++q) w = width[q] > w ? width[q] : w;
  const bool has_in = p->in.host != nullptr;
  const size_t in_bytes = has_in ? (size_t)p->in.rows * w * p->elt : 0;
  const size_t out_bytes = (size_t)p->out.rows * w * p->elt;
  // Three panel slots: panel J + 1 is copied in while J computes and J - 1
  // is still being copied back (with two, J + 1's copy-in waited for J - 1's
  // copy-back, leaving the host-to-device direction idle).
  constexpr int SLOTS = 3;
  void *buf[SLOTS] = {};
  cudaEvent_t ev[SLOTS][3] = {};  // per slot: copied in, computed, copied out
  int st = B200_OK;
  for (int q = 0; q < SLOTS && st == B200_OK; ++q) {
    st = b200_alloc(&buf[q], in_bytes + out_bytes);
    for (int e = 0; e < 3 && st == B200_OK; ++e)
      if (cudaEventCreateWithFlags(&ev[q][e], cudaEventDisableTiming) != cudaSuccess)
        st = b200_set_error(B200_ECUDA, "pipeline: event creation failed");
  }
  cudaEvent_t ready = nullptr;
  if (st == B200_OK && (cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) != cudaSuccess ||
                        cudaEventRecord(ready, sc) != cudaSuccess ||
                        cudaStreamWaitEvent(si, ready, 0) != cudaSuccess))
    st = b200_set_error(B200_ECUDA, "pipeline: stream ordering failed");
  long issued = 0;
  for (int pn = 0; pn < np && st == B200_OK; ++pn, ++issued) {
    const int pq = p->reverse ? np - 1 - pn : pn;
    const long j0 = start[pq], cols = width[pq];
    const int q = (int)(issued % SLOTS);
    char *in_dev = (char *)buf[q], *out_dev = (char *)buf[q] + in_bytes;
    if (issued >= SLOTS) {  // the slot's previous panel has been computed and copied out
      cudaStreamWaitEvent(si, ev[q][1], 0);
      cudaStreamWaitEvent(si, ev[q][2], 0);
    }
    const PanelCopy ci = has_in ? panel_copy(p->in, j0, cols, p->elt) : PanelCopy{};
    const PanelCopy co = panel_copy(p->out, j0, cols, p->elt, p->out_lower ? j0 : 0);
    cudaError_t e = cudaSuccess;
    // The streamed operands' blocks of this panel go first: the panel's
    // arithmetic reads them (and, with reverse, the blocks of the panels
    // to its right, which came earlier on the same stream).
    for (int t = 0; t < p->nstreams && e == cudaSuccess; ++t) {
      const b200_colpipe_stream_t &s = p->streams[t];
      const long r0 = s.by_cols ? 0 : j0, c0 = s.by_cols ? j0 : 0;
      const long nr = s.by_cols ? s.extent : cols, nc = s.by_cols ? cols : s.extent;
      const char *src = (const char *)s.host + (r0 * s.rs + c0 * s.cs) * (long)p->elt;
      char *dst = (char *)s.dev + (r0 * s.drs + c0 * s.dcs) * (long)p->elt;
      if (s.rs == 1 && s.drs == 1)
        e = b200_h2d_2d(dst, s.dcs * p->elt, src, s.cs * p->elt, nr * p->elt, nc, si);
      else
        e = b200_h2d_2d(dst, s.drs * p->elt, src, s.rs * p->elt, nc * p->elt, nr, si);
    }
    if (has_in && e == cudaSuccess)
      e = b200_h2d_2d(in_dev, ci.dpitch, (const char *)p->in.host + ci.off * p->elt, ci.hpitch,
                      ci.width, ci.height, si);
    if (e == cudaSuccess && p->out_read) {
      if (p->out_lower)
        e = lower_panel_copy(p->out, j0, cols, p->elt, out_dev, co, true, si);
      else
        e = b200_h2d_2d(out_dev, co.dpitch, (const char *)p->out.host + co.off * p->elt,
                        co.hpitch, co.width, co.height, si);
    }
    if (e == cudaSuccess) e = cudaEventRecord(ev[q][0], si);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sc, ev[q][0], 0);
    if (e != cudaSuccess) {
      st = b200_set_error(B200_ECUDA, "pipeline: panel copy-in failed");
      break;
    }
    st = p->run(p->ctx, j0, cols, has_in ? in_dev : nullptr, ci.drs, ci.dcs, out_dev, co.drs,
                co.dcs);
    if (st != B200_OK) break;
    e = cudaEventRecord(ev[q][1], sc);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(so, ev[q][1], 0);
    if (e == cudaSuccess)
      e = p->out_lower ? lower_panel_copy(p->out, j0, cols, p->elt, out_dev, co, false, so)
                       : cudaMemcpy2DAsync((char *)p->out.host + co.off * p->elt, co.hpitch,
                                           out_dev, co.dpitch, co.width, co.height,
                                           cudaMemcpyDeviceToHost, so);
    if (e == cudaSuccess) e = cudaEventRecord(ev[q][2], so);
    if (e != cudaSuccess) st = b200_set_error(B200_ECUDA, "pipeline: panel copy-out failed");
  }
  // Drain: the copy streams finish, then the buffers are released on sc.
  cudaStreamSynchronize(si);
  cudaStreamSynchronize(so);
  const int sync = b200_stream_sync();
  for (int q = 0; q < SLOTS; ++q) {
    b200_free(buf[q]);
    for (int e = 0; e < 3; ++e)
      if (ev[q][e]) cudaEventDestroy(ev[q][e]);
  }
  if (ready) cudaEventDestroy(ready);
  return st != B200_OK ? st : sync;
}

// ---- public runtime controls (include/mublis_b200.h) ----------------------

int mublis_b200_init(void) { return b200_init(); }

const char *mublis_b200_last_error(void) { return b200_last_error(); }

int mublis_b200_set_stream(void *stream) {
  B200_TRY(b200_init());
  return b200_set_thread_stream(stream);
}

void *mublis_b200_get_stream(void) {
  if (b200_init() != B200_OK) return nullptr;
  return b200_stream();
}

int mublis_b200_set_form(char dtype, const char *form) {
  B200_TRY(b200_init());
  int slices = 0;
  double target = 0.0;
  int f = b200_parse_form(form, &slices, &target);
  if (f == B200_FORM_AUTO) return B200_EINVAL;
  const int dt = dtype == 'd' ? B200_F64 : B200_F32;
  B200_TRY(b200_set_default_form(dt, f, slices));
  if (f == B200_FORM_OZAKI2) g_default_target[dt == B200_F64] = target;
  return B200_OK;
}

unsigned long long mublis_b200_launch_count(void) { return g_launches.load(); }

int mublis_b200_profile_enable(int on) {
  g_prof_on.store(on ? 1 : 0);
  return B200_OK;
}

// Writes {"kernel": [launches, total_ms], ...} for every launch recorded
// since the last read, then forgets them.  Synchronises the device.
int mublis_b200_profile_read(char *buf, unsigned long len) {
  cudaDeviceSynchronize();
  std::vector<ProfRec> recs;
  {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    recs.swap(g_prof);
  }
  std::vector<std::pair<std::string, std::pair<int, double>>> agg;
  for (auto &r : recs) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.start, r.stop);
    cudaEventDestroy(r.start);
    cudaEventDestroy(r.stop);
    bool found = false;
    for (auto &a : agg)
      if (a.first == r.name) {
        a.second.first += 1;
        a.second.second += ms;
        found = true;
      }
    if (!found) agg.push_back({r.name, {1, (double)ms}});
  }
  std::string out = "{";
  for (size_t i = 0; i < agg.size(); ++i) {
    char tmp[256];
    snprintf(tmp, sizeof tmp, "%s\"%s\": [%d, %.6f]", i ? ", " : "", agg[i].first.c_str(),
             agg[i].second.first, agg[i].second.second);
    out += tmp;
  }
  out += "}";
  if (buf && len) {
    strncpy(buf, out.c_str(), len - 1);
    buf[len - 1] = 0;
  }
  return (int)out.size();
}

}  // extern "C"
