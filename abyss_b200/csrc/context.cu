// Context, buffers, launch planning and the status-returning C ABI
// (include/abyss_reg.h).
//
// The reference keeps its device state in file-static globals sized by
// new_size(N) and reallocated on growth (src_mpi/cuda/cuda_my_acceleration.cu:
// 603-778) and launches compute_forces -> reduce_forces_kernel ->
// gather_neighbor -> gather_numneighbor (:158-218).  Here a context owns
// growable device buffers and one stream; a launch is
//   [target ordering] -> force kernel (tile or j-major) -> finalize
// all enqueued on the context stream.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <string>
#include <vector>

#include "../../include/abyss_reg.h"
#include "abyss_internal.cuh"
#include "ctx_internal.h"
#include "kernels.cuh"

using namespace abyss;

namespace {

template <class T>
struct DevBuf {
  T *p = nullptr;
  size_t cap = 0;  // elements
  cudaError_t ensure(size_t n) {
    if (n <= cap && p) return cudaSuccess;
    // a buffer that has to grow grows by at least half again, so a context
    // that sees slowly rising sizes reallocates (and synchronizes the device
    // in cudaFree) only a few times
    size_t want = std::max<size_t>(std::max<size_t>(n, 1), cap + cap / 2);
    want = (want + kPad - 1) / kPad * kPad;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void **)&p, want * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    cap = want;
    return cudaSuccess;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// Pinned host memory for the copies of one call between pageable caller
// memory and the device.  The driver copies pageable memory through its own
// staging, which serialises such copies across host threads and waits for the
// device; copies through a context's own pinned buffer are plain DMA.
struct HostStage {
  unsigned char *p = nullptr;
  size_t cap = 0;  // bytes
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    const size_t want = std::max(bytes, cap + cap / 2);
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaHostAlloc((void **)&p, want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
      p = nullptr;
      return e;
    }
    cap = want;
    return cudaSuccess;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

// Pageable copies larger than this go the driver's way, which overlaps its
// host-side staging with the DMA.
constexpr size_t kStageMax = (size_t)16 << 20;

struct Table {
  std::vector<int> m_max;
  std::vector<abyss_tuning> entries;
};

}  // namespace

struct abyss_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  std::string err;
  // j-set
  int n = 0;
  bool have_state = false, have_jset = false;
  DevBuf<double> x, v, a0, a1, t0, mass, r2nb;           // state (AoS for vectors)
  DevBuf<double> px, py, pz, pvx, pvy, pvz;              // predicted SoA
  DevBuf<float4> vm;
  // targets and ordering
  int m = 0;
  DevBuf<int> targets, order_t, order_o, iota, rows, rows_alt, bbox;
  DevBuf<uint32_t> keys, keys_alt;
  DevBuf<double> anchor;  // anchor mode: [i-blocks][3] bounding-box centres
  DevBuf<char> cub_tmp;
  size_t cub_bytes = 0;
  // per-launch work and outputs
  DevBuf<int> lcnt, lst, status, ovf, items, ovf_list;
  DevBuf<double> part;
  DevBuf<double> acc_reg, jerk_reg, acc_irr, jerk_irr;
  DevBuf<int> nnb, list;
  int launched_m = 0, launched_cap = 0;
  bool launched = false;
  abyss_tuning plan{};
  int plan_chunks = 0;
  Table table;
  // profiling: 0 off, 1 each phase, 2 the whole launch (two events)
  int profiling = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // host waits: < 0 stream synchronisation, else spin this long, then block
  int wait_spin_us = -1;
  cudaEvent_t ev_wait = nullptr;  // cudaEventBlockingSync
  // pinned staging of pageable caller memory: inputs, and results; ev_hin
  // marks the end of the last copies out of `hin`
  HostStage hin, hout;
  cudaEvent_t ev_hin = nullptr;
  // scratch for energies
  DevBuf<double> e_x, e_v, e_m, e_row;
  DevBuf<double> i_a0, i_a1, i_r2, i_out;  // initialisation derivatives
};

static int fail(abyss_ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  return code;
}

static int cuda_fail(abyss_ctx *c, cudaError_t e, const char *what) {
  return fail(c, e == cudaErrorMemoryAllocation ? ABYSS_ERR_OOM : ABYSS_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

// Wait on the host for everything queued on the context stream.  By default
// this is the stream synchronisation, whose waiting thread keeps its core (it
// spins while the process has no more threads than cores).  With a wait policy
// (abyss_set_wait) the thread polls for at most wait_spin_us and then sleeps in
// a blocking event wait, leaving its core to other host threads while the GPU
// is busy with other work.
static cudaError_t ctx_wait(abyss_ctx *c) {
  if (c->wait_spin_us < 0 || !c->ev_wait) return cudaStreamSynchronize(c->stream);
  cudaError_t e = cudaEventRecord(c->ev_wait, c->stream);
  if (e != cudaSuccess) return e;
  const auto t0 = std::chrono::steady_clock::now();
  const auto spin = std::chrono::microseconds(c->wait_spin_us);
  for (;;) {
    e = cudaEventQuery(c->ev_wait);
    if (e != cudaErrorNotReady) return e;
    if (std::chrono::steady_clock::now() - t0 >= spin) break;
  }
  return cudaEventSynchronize(c->ev_wait);
}

// Wait for `ev` (created with cudaEventBlockingSync) by the context's policy.
static cudaError_t wait_event(abyss_ctx *c, cudaEvent_t ev) {
  const auto t0 = std::chrono::steady_clock::now();
  const auto spin = std::chrono::microseconds(std::max(c->wait_spin_us, 0));
  for (;;) {
    const cudaError_t e = cudaEventQuery(ev);
    if (e != cudaErrorNotReady) return e;
    if (c->wait_spin_us >= 0 && std::chrono::steady_clock::now() - t0 >= spin) break;
  }
  return cudaEventSynchronize(ev);
}

static bool host_pinned(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

static size_t round16(size_t b) { return (b + 15) & ~(size_t)15; }

// One host<->device copy of a call.
struct Xfer {
  void *dst;
  const void *src;
  size_t bytes;
};

// Queue the host-to-device copies of one call.  Pinned sources are copied
// directly; pageable ones (up to kStageMax in all) through `hin`, after the
// copies that last read it have finished.
static cudaError_t h2d(abyss_ctx *c, std::initializer_list<Xfer> xs) {
  if (xs.size() > 16) return cudaErrorInvalidValue;
  bool stage[16];
  size_t need = 0, k = 0;
  for (const Xfer &x : xs) {
    stage[k] = x.bytes > 0 && !host_pinned(x.src);
    if (stage[k]) need += round16(x.bytes);
    ++k;
  }
  const bool staged = need > 0 && need <= kStageMax;
  if (staged) {
    cudaError_t e = wait_event(c, c->ev_hin);
    if (e == cudaSuccess) e = c->hin.ensure(need);
    if (e != cudaSuccess) return e;
  }
  size_t off = 0;
  k = 0;
  for (const Xfer &x : xs) {
    const void *src = x.src;
    if (staged && stage[k]) {
      std::memcpy(c->hin.p + off, x.src, x.bytes);
      src = c->hin.p + off;
      off += round16(x.bytes);
    }
    ++k;
    if (x.bytes == 0) continue;
    const cudaError_t e = cudaMemcpyAsync(x.dst, src, x.bytes, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return e;
  }
  return staged ? cudaEventRecord(c->ev_hin, c->stream) : cudaSuccess;
}

// The device-to-host copies of one call: queue() them (pageable destinations,
// up to kStageMax in all, into `hout`), wait for the stream, then finish()
// copies the staged bytes to their destinations.
struct D2H {
  std::vector<Xfer> out;  // staged: dst = caller memory, src = hout
  cudaError_t queue(abyss_ctx *c, std::initializer_list<Xfer> xs) {
    if (xs.size() > 16) return cudaErrorInvalidValue;
    size_t need = 0;
    bool stage[16];
    size_t k = 0;
    for (const Xfer &x : xs) {
      stage[k] = x.bytes > 0 && !host_pinned(x.dst);
      if (stage[k]) need += round16(x.bytes);
      ++k;
    }
    const bool staged = need > 0 && need <= kStageMax;
    if (staged) {
      // the previous call's results were read out before it returned
      cudaError_t e = c->hout.ensure(need);
      if (e != cudaSuccess) return e;
    }
    size_t off = 0;
    k = 0;
    for (const Xfer &x : xs) {
      void *dst = x.dst;
      if (staged && stage[k]) {
        dst = c->hout.p + off;
        out.push_back(Xfer{x.dst, dst, x.bytes});
        off += round16(x.bytes);
      }
      ++k;
      if (x.bytes == 0) continue;
      const cudaError_t e = cudaMemcpyAsync(dst, x.src, x.bytes, cudaMemcpyDeviceToHost, c->stream);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
  void finish() {
    for (const Xfer &x : out) std::memcpy(x.dst, x.src, x.bytes);
  }
};

#define CK(expr, what)                                  \
  do {                                                  \
    cudaError_t _e = (expr);                            \
    if (_e != cudaSuccess) return cuda_fail(c, _e, what); \
  } while (0)

static JSet jset_of(abyss_ctx *c) {
  JSet js;
  js.px = c->px.p;
  js.py = c->py.p;
  js.pz = c->pz.p;
  js.vm = c->vm.p;
  js.pvx = c->pvx.p;
  js.pvy = c->pvy.p;
  js.pvz = c->pvz.p;
  js.mass = c->mass.p;
  js.r2nb = c->r2nb.p;
  js.n = c->n;
  return js;
}

static int ensure_jset(abyss_ctx *c, int n) {
  const size_t n1 = (size_t)n + 2;  // slack for the even-count bulk copies
  CK(c->px.ensure(n1), "alloc px");
  CK(c->py.ensure(n1), "alloc py");
  CK(c->pz.ensure(n1), "alloc pz");
  CK(c->pvx.ensure(n1), "alloc pvx");
  CK(c->pvy.ensure(n1), "alloc pvy");
  CK(c->pvz.ensure(n1), "alloc pvz");
  CK(c->vm.ensure(n1), "alloc vm");
  CK(c->mass.ensure(n1), "alloc mass");
  CK(c->r2nb.ensure(n1), "alloc r2nb");
  return ABYSS_OK;
}

static int ensure_targets(abyss_ctx *c, int m) {
  CK(c->targets.ensure(m), "alloc targets");
  CK(c->order_t.ensure(m), "alloc order_t");
  CK(c->order_o.ensure(m), "alloc order_o");
  if (c->iota.cap < (size_t)m) {
    CK(c->iota.ensure(m), "alloc iota");
    launch_iota(c->stream, (int)c->iota.cap, c->iota.p, c->sm_count);
  }
  return ABYSS_OK;
}

static int ensure_outputs(abyss_ctx *c, int m, int cap) {
  CK(c->acc_reg.ensure((size_t)3 * m), "alloc acc_reg");
  CK(c->jerk_reg.ensure((size_t)3 * m), "alloc jerk_reg");
  CK(c->acc_irr.ensure((size_t)3 * m), "alloc acc_irr");
  CK(c->jerk_irr.ensure((size_t)3 * m), "alloc jerk_irr");
  CK(c->nnb.ensure(m), "alloc nnb");
  CK(c->list.ensure((size_t)m * cap), "alloc list");
  CK(c->status.ensure(1), "alloc status");
  CK(c->ovf.ensure(1), "alloc ovf");
  return ABYSS_OK;
}

namespace abyss {
// accessors used by the batched-ensemble layer (ensemble.cu)
cudaStream_t ctx_stream(abyss_ctx *c) { return c->stream; }
int ctx_device(abyss_ctx *c) { return c->device; }
int ctx_sm_count(abyss_ctx *c) { return c->sm_count; }
int ctx_wait_spin(abyss_ctx *c) { return c->wait_spin_us; }

// ---- used by whole regular blocks on the device (host/ac_integrator.cpp):
// the state the host would upload is written into the context by a kernel on
// its stream, the targets come from device memory, and the results stay there.

// Device arrays of the j-set state for n particles, to be written on the
// context stream before abyss_predict (as abyss_upload_state would).
int ctx_state_buffers(abyss_ctx *c, int n, abyss_irr::JsetDst *d) {
  if (!c || n <= 0 || !d) return ABYSS_ERR_ARG;
  cudaSetDevice(c->device);
  int rc = ensure_jset(c, n);
  if (rc != ABYSS_OK) return rc;
  const size_t v3 = (size_t)3 * n;
  CK(c->x.ensure(v3), "alloc x");
  CK(c->v.ensure(v3), "alloc v");
  CK(c->a0.ensure(v3), "alloc a0");
  CK(c->a1.ensure(v3), "alloc a1");
  CK(c->t0.ensure(n), "alloc t0");
  *d = abyss_irr::JsetDst{c->x.p, c->v.p, c->a0.p, c->a1.p, c->t0.p, c->mass.p, c->r2nb.p};
  c->n = n;
  c->have_state = true;
  c->have_jset = false;
  return ABYSS_OK;
}

// m targets copied on the context stream from device memory (indices already
// inside the j-set: they come from the integrator's own scheduling kernel).
int ctx_targets_from_device(abyss_ctx *c, int m, const int *d_targets) {
  if (!c || m <= 0 || !d_targets) return ABYSS_ERR_ARG;
  if (c->n <= 0 || m > c->n) return fail(c, ABYSS_ERR_STATE, "targets: no j-set of that size");
  cudaSetDevice(c->device);
  int rc = ensure_targets(c, m);
  if (rc != ABYSS_OK) return rc;
  CK(cudaMemcpyAsync(c->targets.p, d_targets, sizeof(int) * (size_t)m, cudaMemcpyDeviceToDevice, c->stream),
     "D2D targets");
  c->m = m;
  return ABYSS_OK;
}

// The last launch's status word and overflowed-row count (waits for it).
int ctx_launch_status(abyss_ctx *c, int *status, int *ovf) {
  if (!c || !status || !ovf) return ABYSS_ERR_ARG;
  if (!c->launched) return fail(c, ABYSS_ERR_STATE, "status: nothing launched");
  cudaSetDevice(c->device);
  int st = 0, ov = 0;
  D2H out;  // through the pinned staging: many host threads wait on one GPU
  CK(out.queue(c, {{&st, c->status.p, sizeof(int)}, {&ov, c->ovf.p, sizeof(int)}}), "D2H status");
  CK(ctx_wait(c), "synchronize");
  out.finish();
  *status = st & kErrTimeout ? ABYSS_ERR_TIMEOUT : ABYSS_OK;
  *ovf = ov;
  return ABYSS_OK;
}

// Device pointers of the last launch's results.
int ctx_results(abyss_ctx *c, abyss_irr::RegResults *r) {
  if (!c || !r) return ABYSS_ERR_ARG;
  if (!c->launched) return fail(c, ABYSS_ERR_STATE, "results: nothing launched");
  *r = abyss_irr::RegResults{c->acc_reg.p, c->jerk_reg.p, c->acc_irr.p, c->jerk_irr.p, c->nnb.p, c->list.p,
                             c->launched_cap};
  return ABYSS_OK;
}

// The last launch's targets (m) and the j-set radii (n), into host memory.
int ctx_read_targets(abyss_ctx *c, int *targets, double *r2nb) {
  if (!c) return ABYSS_ERR_ARG;
  if (!c->launched) return fail(c, ABYSS_ERR_STATE, "read targets: nothing launched");
  cudaSetDevice(c->device);
  D2H out;
  CK(out.queue(c, {{targets, c->targets.p, targets ? sizeof(int) * (size_t)c->launched_m : 0},
                   {r2nb, c->r2nb.p, r2nb ? sizeof(double) * (size_t)c->n : 0}}),
     "D2H targets and radii");
  CK(ctx_wait(c), "synchronize");
  out.finish();
  return ABYSS_OK;
}
}  // namespace abyss

extern "C" {

int abyss_create(int device, abyss_ctx **out) {
  if (!out) return ABYSS_ERR_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) return ABYSS_ERR_NODEVICE;
  if (device < 0 || device >= count) return ABYSS_ERR_ARG;
  abyss_ctx *c = new abyss_ctx;
  c->device = device;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreate(&c->ev[i]);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_hin, cudaEventBlockingSync | cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(c->ev_hin, c->stream);
  if (e != cudaSuccess) {
    delete c;
    return ABYSS_ERR_CUDA;
  }
  *out = c;
  return ABYSS_OK;
}

int abyss_destroy(abyss_ctx *c) {
  if (!c) return ABYSS_ERR_ARG;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  DevBuf<double> *dbl[] = {&c->anchor, &c->x, &c->v, &c->a0, &c->a1, &c->t0, &c->mass, &c->r2nb, &c->px, &c->py,
                           &c->pz, &c->pvx, &c->pvy, &c->pvz, &c->part, &c->acc_reg, &c->jerk_reg,
                           &c->acc_irr, &c->jerk_irr, &c->e_x, &c->e_v, &c->e_m, &c->e_row,
                           &c->i_a0, &c->i_a1, &c->i_r2, &c->i_out};
  for (auto *b : dbl) b->release();
  DevBuf<int> *ints[] = {&c->targets, &c->order_t, &c->order_o, &c->iota, &c->rows, &c->rows_alt,
                         &c->bbox, &c->lcnt, &c->lst, &c->status, &c->ovf, &c->nnb, &c->list,
                         &c->items, &c->ovf_list};
  for (auto *b : ints) b->release();
  c->vm.release();
  c->keys.release();
  c->keys_alt.release();
  c->cub_tmp.release();
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->ev_wait) cudaEventDestroy(c->ev_wait);
  if (c->ev_hin) cudaEventDestroy(c->ev_hin);
  c->hin.release();
  c->hout.release();
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return ABYSS_OK;
}

const char *abyss_last_error(const abyss_ctx *c) { return c ? c->err.c_str() : "null context"; }

void *abyss_stream(abyss_ctx *c) { return c ? (void *)c->stream : nullptr; }

int abyss_synchronize(abyss_ctx *c) {
  if (!c) return ABYSS_ERR_ARG;
  cudaSetDevice(c->device);
  CK(ctx_wait(c), "synchronize");
  return ABYSS_OK;
}

int abyss_set_wait(abyss_ctx *c, int spin_us) {
  if (!c) return ABYSS_ERR_ARG;
  cudaSetDevice(c->device);
  if (spin_us >= 0 && !c->ev_wait)
    CK(cudaEventCreateWithFlags(&c->ev_wait, cudaEventBlockingSync | cudaEventDisableTiming), "wait event");
  c->wait_spin_us = spin_us < 0 ? -1 : spin_us;
  return ABYSS_OK;
}

int abyss_reserve(abyss_ctx *c, int n, int m, int list_cap) {
  if (!c || n < 0 || m < 0 || list_cap < 0) return fail(c, ABYSS_ERR_ARG, "reserve: negative size");
  cudaSetDevice(c->device);
  int rc;
  if ((rc = ensure_jset(c, n)) != ABYSS_OK) return rc;
  const int m1 = std::max(m, 1), cap1 = std::max(list_cap, 1);
  if ((rc = ensure_targets(c, m1)) != ABYSS_OK) return rc;
  if ((rc = ensure_outputs(c, m1, cap1)) != ABYSS_OK) return rc;
  // un-predicted state, energy and initialisation buffers for n particles
  const size_t n3 = (size_t)3 * std::max(n, 1);
  DevBuf<double> *st[] = {&c->x, &c->v, &c->a0, &c->a1, &c->e_x, &c->e_v, &c->i_a0, &c->i_a1};
  for (auto *b : st) CK(b->ensure(n3), "alloc state");
  DevBuf<double> *st1[] = {&c->t0, &c->e_m, &c->e_row, &c->i_r2};
  for (auto *b : st1) CK(b->ensure(std::max(n, 1)), "alloc state");
  CK(c->i_out.ensure((size_t)12 * std::max(n, 1)), "alloc init");
  // work buffers of the tile kernel: chunk partials for at most the chunk count
  // a launch plan can choose (<= n / 1024 chunks, and <= 32 items per CTA of a
  // grid of at most 8 CTAs per SM over i-blocks of >= 128 targets)
  const int s_items = (int)((32LL * 8 * c->sm_count) / std::max(1, (m1 + 127) / 128)) + 1;
  const int s_max = std::max(1, std::min((std::max(n, 1) + 1023) / 1024, s_items));
  CK(c->lcnt.ensure((size_t)m1), "alloc lcnt");
  CK(c->lst.ensure((size_t)m1 * cap1), "alloc lst");
  CK(c->part.ensure((size_t)s_max * m1 * 6), "alloc part");
  CK(c->items.ensure(1), "alloc items");
  CK(c->ovf_list.ensure((size_t)m1), "alloc overflow list");
  // pinned staging for pageable callers: the state upload (15 doubles per
  // particle) and the targets; the results (12 doubles and 1 + list_cap ints
  // per target) or the initialisation derivatives (12 doubles per particle)
  const size_t n1 = std::max(n, 1);
  const size_t in_b = 15 * 8 * n1 + 4 * (size_t)m1 + 16 * 16;
  const size_t out_b = std::max(96 * n1, (96 + 4 + 4 * (size_t)cap1) * m1) + 16 * 16;
  CK(wait_event(c, c->ev_hin), "staging");
  CK(c->hin.ensure(std::min(in_b, kStageMax)), "pinned staging");
  CK(c->hout.ensure(std::min(out_b, kStageMax)), "pinned staging");
  return ABYSS_OK;
}

int abyss_upload_state(abyss_ctx *c, int n, const double *x, const double *v, const double *a0,
                       const double *a1, const double *t0, const double *mass, const double *r2nb) {
  if (!c) return ABYSS_ERR_ARG;
  if (n <= 0 || !x || !v || !a0 || !a1 || !t0 || !mass || !r2nb)
    return fail(c, ABYSS_ERR_ARG, "upload_state: n <= 0 or null array");
  cudaSetDevice(c->device);
  int rc = ensure_jset(c, n);
  if (rc != ABYSS_OK) return rc;
  const size_t v3 = (size_t)3 * n;
  CK(c->x.ensure(v3), "alloc x");
  CK(c->v.ensure(v3), "alloc v");
  CK(c->a0.ensure(v3), "alloc a0");
  CK(c->a1.ensure(v3), "alloc a1");
  CK(c->t0.ensure(n), "alloc t0");
  CK(h2d(c, {{c->x.p, x, v3 * 8}, {c->v.p, v, v3 * 8}, {c->a0.p, a0, v3 * 8}, {c->a1.p, a1, v3 * 8},
             {c->t0.p, t0, (size_t)n * 8}, {c->mass.p, mass, (size_t)n * 8}, {c->r2nb.p, r2nb, (size_t)n * 8}}),
     "H2D state");
  c->n = n;
  c->have_state = true;
  c->have_jset = false;
  return ABYSS_OK;
}

int abyss_predict(abyss_ctx *c, double new_time, double time_scale) {
  if (!c) return ABYSS_ERR_ARG;
  if (!c->have_state) return fail(c, ABYSS_ERR_STATE, "predict: no state uploaded");
  cudaSetDevice(c->device);
  launch_predict(c->stream, c->n, c->x.p, c->v.p, c->a0.p, c->a1.p, c->t0.p, c->mass.p, new_time,
                 time_scale, c->px.p, c->py.p, c->pz.p, c->pvx.p, c->pvy.p, c->pvz.p, c->vm.p,
                 c->sm_count);
  CK(cudaGetLastError(), "predict launch");
  c->have_jset = true;
  return ABYSS_OK;
}

int abyss_upload_predicted(abyss_ctx *c, int n, const double *px, const double *pv,
                           const double *mass, const double *r2nb) {
  if (!c) return ABYSS_ERR_ARG;
  if (n <= 0 || !px || !pv || !mass || !r2nb)
    return fail(c, ABYSS_ERR_ARG, "upload_predicted: n <= 0 or null array");
  cudaSetDevice(c->device);
  int rc = ensure_jset(c, n);
  if (rc != ABYSS_OK) return rc;
  const size_t v3 = (size_t)3 * n;
  CK(c->x.ensure(v3), "alloc x");
  CK(c->v.ensure(v3), "alloc v");
  CK(h2d(c, {{c->x.p, px, v3 * 8}, {c->v.p, pv, v3 * 8}, {c->mass.p, mass, (size_t)n * 8},
             {c->r2nb.p, r2nb, (size_t)n * 8}}),
     "H2D predicted");
  launch_unpack_predicted(c->stream, n, c->x.p, c->v.p, c->mass.p, c->px.p, c->py.p, c->pz.p,
                          c->pvx.p, c->pvy.p, c->pvz.p, c->vm.p, c->sm_count);
  CK(cudaGetLastError(), "unpack launch");
  c->n = n;
  c->have_state = false;
  c->have_jset = true;
  return ABYSS_OK;
}

int abyss_read_predicted(abyss_ctx *c, double *px, double *pv, float *vm4) {
  if (!c) return ABYSS_ERR_ARG;
  if (!c->have_jset) return fail(c, ABYSS_ERR_STATE, "read_predicted: no predicted j-set");
  cudaSetDevice(c->device);
  const size_t n = c->n;
  std::vector<double> tmp(6 * n);
  double *dst[6] = {tmp.data(), tmp.data() + n, tmp.data() + 2 * n,
                    tmp.data() + 3 * n, tmp.data() + 4 * n, tmp.data() + 5 * n};
  const double *src[6] = {c->px.p, c->py.p, c->pz.p, c->pvx.p, c->pvy.p, c->pvz.p};
  D2H out;
  CK(out.queue(c, {{dst[0], src[0], n * 8}, {dst[1], src[1], n * 8}, {dst[2], src[2], n * 8},
                   {dst[3], src[3], n * 8}, {dst[4], src[4], n * 8}, {dst[5], src[5], n * 8},
                   {vm4, c->vm.p, vm4 ? n * 16 : 0}}),
     "D2H predicted");
  CK(ctx_wait(c), "synchronize");
  out.finish();
  for (size_t j = 0; j < n; ++j)
    for (int d = 0; d < 3; ++d) {
      if (px) px[3 * j + d] = dst[d][j];
      if (pv) pv[3 * j + d] = dst[3 + d][j];
    }
  return ABYSS_OK;
}

int abyss_set_targets(abyss_ctx *c, int m, const int *targets) {
  if (!c) return ABYSS_ERR_ARG;
  if (m <= 0 || !targets) return fail(c, ABYSS_ERR_ARG, "set_targets: m <= 0 or null targets");
  if (c->n <= 0) return fail(c, ABYSS_ERR_STATE, "set_targets: no j-set uploaded");
  if (m > c->n) return fail(c, ABYSS_ERR_ARG, "set_targets: m > n");
  for (int k = 0; k < m; ++k)
    if (targets[k] < 0 || targets[k] >= c->n)
      return fail(c, ABYSS_ERR_ARG, "set_targets: target index out of range");
  cudaSetDevice(c->device);
  int rc = ensure_targets(c, m);
  if (rc != ABYSS_OK) return rc;
  CK(h2d(c, {{c->targets.p, targets, (size_t)m * 4}}), "H2D targets");
  c->m = m;
  return ABYSS_OK;
}

// ------------------------------------------------------------------ planning
// Launches of at most this many rows on the j-major kernel finalize in the force
// kernel's last block instead of a second launch.
constexpr int kFuseRows = 2;

static abyss_tuning plan_for(abyss_ctx *c, int m, const abyss_tuning *user) {
  abyss_tuning t{};
  if (user) t = *user;
  if (t.kernel == 0) {
    for (size_t k = 0; k < c->table.m_max.size(); ++k)
      if (m <= c->table.m_max[k]) {
        const abyss_tuning &e = c->table.entries[k];
        if (t.kernel == 0) t.kernel = e.kernel;
        if (t.mode == 0) t.mode = e.mode;
        if (t.threads == 0) t.threads = e.threads;
        if (t.ipt == 0) t.ipt = e.ipt;
        if (t.j_split == 0) t.j_split = e.j_split;
        if (t.grid == 0) t.grid = e.grid;
        if (t.unroll == 0) t.unroll = e.unroll;
        if (t.min_blocks == 0) t.min_blocks = e.min_blocks;
        break;
      }
  }
  // Built-in rule (measured on B200, King W0=6, N = 2^20): lanes over j for
  // tiny active sets; warps sharing targets up to 96; one target per thread on
  // the scalar tile kernel in 128-thread blocks up to 128 targets (or 32/64-thread
  // blocks when a tuning asks for them); otherwise the packed
  // tile kernel, with anchor offsets on Hilbert-ordered targets once the active
  // set is dense enough for them to be accurate, double-single offsets below
  // that.
  if (t.kernel == 0) {
    if (m <= 20) {
      t.kernel = 2;
    } else if (m <= 128 && t.threads == 0 && t.ipt == 0 && (t.mode == 0 || t.mode == 2)) {
      // 21-128 targets: the block's 4 warps share 32 (or 64) targets and
      // split each j-tile.  Measured whole calls (Gpairs/s): m = 24 packed
      // over two j 304 (j-major 277); m = 32 the same 406 (scalar with two j
      // per step 385); m = 48 scalar 346 (packed 333); m = 64 packed over a
      // thread's two targets 551 (scalar 487); m = 96 scalar 524 (packed
      // 492); m = 128 packed, two targets 605 (one target per thread on the
      // 128-thread tile kernel 592)
      if (m <= 32) {
        t.kernel = 5;
        t.ipt = 1;
        if (t.j_split == 0) t.j_split = 1024;
      } else if (m <= 48 || (m > 64 && m <= 96)) {
        t.kernel = 4;
        t.ipt = 1;
        t.unroll = 2;
        if (t.j_split == 0) t.j_split = m <= 48 ? 2048 : 1024;
      } else {
        t.kernel = 5;
        t.ipt = 2;
        if (t.j_split == 0) t.j_split = 1024;
      }
    } else if (m <= 128 && (t.threads == 0 || t.threads == (m <= 48 ? 32 : m <= 96 ? 64 : 128)) &&
               (t.ipt == 0 || t.ipt == 1) && (t.mode == 0 || t.mode == 2)) {
      t.kernel = 1;
      t.mode = 2;
      t.threads = m <= 48 ? 32 : m <= 96 ? 64 : 128;
      t.ipt = 1;
      if (t.j_split == 0) t.j_split = t.threads == 32 ? 1024 : t.threads == 64 ? 4096 : 2048;
    } else {
      t.kernel = 3;
    }
  }
  if (t.kernel == 2) {
    if (t.ipt == 0) t.ipt = m <= 1 ? 1 : m <= 2 ? 2 : m <= 4 ? 4 : 8;
  } else if (t.kernel == 3) {
    if (t.mode == 0) t.mode = (m >= 16384) ? 1 : 2;
    // measured on B200 (King W0=6, N = 2^20): anchor 128 threads x 6 targets,
    // 3 CTAs per SM (168 registers); double-single 128 x 4 with 2 j per step,
    // 4 CTAs per SM, or, for active sets too small to fill 512-target blocks,
    // 128 x 2 with 1 j per step at 5 CTAs per SM (2048 j-chunks up to 256
    // targets)
    if (t.mode == 1) {
      if (t.threads == 0) t.threads = 128;
      if (t.ipt == 0) t.ipt = 6;
      if (t.unroll == 0 && t.threads == 128 && (t.ipt == 6 || t.ipt == 8)) t.unroll = 1;
      if (t.min_blocks == 0 && t.threads == 128 && t.ipt == 6) t.min_blocks = 3;
      if (t.min_blocks == 0 && t.threads == 128 && t.ipt == 8) t.min_blocks = 2;
    } else {
      if (t.threads == 0) t.threads = 128;
      if (t.ipt == 0) t.ipt = (m >= 1024) ? 4 : 2;
      if (t.threads == 128 && t.ipt == 4) {
        if (t.unroll == 0) t.unroll = 2;
        if (t.min_blocks == 0) t.min_blocks = 4;
      } else if (t.threads == 128 && t.ipt == 2 && t.unroll == 0 && t.min_blocks == 0) {
        t.unroll = 1;
        t.min_blocks = 5;
        if (t.j_split == 0 && m <= 256) t.j_split = 2048;
      }
    }
  } else if (t.kernel == 4 || t.kernel == 5) {
    // warps sharing targets: 4 warps, double-single offsets, 32 x ipt targets
    // per block (kernel 5: packed FP32x2 arithmetic, one j per step for ipt 1
    // -- its two halves are two j)
    t.mode = 2;
    t.threads = 128;
    if (t.ipt == 0) t.ipt = 1;
    if (t.unroll == 0 || (t.kernel == 5 && t.ipt == 1)) t.unroll = 1;
    t.min_blocks = 1;
  } else {
    if (t.mode == 0) t.mode = (m >= 4096) ? 1 : 2;
    if (t.threads == 0) t.threads = 128;
    if (t.ipt == 0) t.ipt = (m >= 65536) ? 2 : 1;
  }
  return t;
}

int abyss_launch(abyss_ctx *c, double eps2, int list_cap, const abyss_tuning *tuning) {
  if (!c) return ABYSS_ERR_ARG;
  if (!c->have_jset) return fail(c, ABYSS_ERR_STATE, "launch: no predicted j-set");
  if (c->m <= 0) return fail(c, ABYSS_ERR_STATE, "launch: no targets");
  if (list_cap <= 0) return fail(c, ABYSS_ERR_ARG, "launch: list_cap must be positive");
  if (!(eps2 >= 0.0)) return fail(c, ABYSS_ERR_ARG, "launch: eps2 must be >= 0");
  cudaSetDevice(c->device);
  const int n = c->n, m = c->m;
  abyss_tuning t = plan_for(c, m, tuning);
  constexpr int TJ = 128;
  int S = 1, L = 0, grid = 0, n_iblocks = 0;
  if (t.kernel == 2) {
    if (t.ipt != 1 && t.ipt != 2 && t.ipt != 4 && t.ipt != 8)
      return fail(c, ABYSS_ERR_ARG, "launch: j-major ipt must be 1, 2, 4 or 8");
    // j_split counts j-chunks, one block of jmajor_warps() warps each; by
    // default as many blocks as fit on the GPU at once
    const int nw = jmajor_warps();
    const int want = t.j_split > 0 ? t.j_split : c->sm_count * jmajor_occupancy(t.ipt);
    L = (n + want * nw - 1) / (want * nw);
    L = std::max(64, (L + 63) / 64 * 64);
    S = (n + L * nw - 1) / (L * nw);
  } else if (t.kernel == 1 || t.kernel == 3 || t.kernel == 4 || t.kernel == 5) {
    const bool split = t.kernel == 4 || t.kernel == 5;
    const int per_block = split ? 32 * t.ipt : t.threads * t.ipt;
    n_iblocks = (m + per_block - 1) / per_block;
    const int occ = split ? tile_split_occupancy(t.ipt, t.unroll, t.kernel == 5)
                                  : tile_occupancy(t.threads, t.ipt, t.mode == 1, t.kernel == 3, t.unroll, t.min_blocks);
    if (occ <= 0) return fail(c, ABYSS_ERR_ARG, "launch: unsupported tile shape");
    // persistent grid: every SM holds the same number of CTAs, which take
    // (i-block, j-chunk) items from a device counter
    grid = t.grid > 0 ? t.grid : occ * c->sm_count;
    int s_want = t.j_split;
    if (s_want <= 0) s_want = std::max(1, (32 * grid + n_iblocks - 1) / n_iblocks);
    const int max_chunks = std::max(1, (n + 8 * TJ - 1) / (8 * TJ));
    if (t.j_split <= 0) s_want = std::min(s_want, max_chunks);
    s_want = std::min(s_want, std::max(1, (n + TJ - 1) / TJ));
    int chunk = (n + s_want - 1) / s_want;
    chunk = (chunk + TJ - 1) / TJ * TJ;
    L = chunk;
    S = (n + chunk - 1) / chunk;
    grid = std::min(grid, n_iblocks * S);
    // TMA bulk copies start at multiples of the chunk length: keep it even
    if (L % 2 != 0) return fail(c, ABYSS_ERR_STATE, "launch: j-chunk length must be even");
  } else {
    return fail(c, ABYSS_ERR_ARG, "launch: unknown kernel");
  }
  if (list_cap > 8192) return fail(c, ABYSS_ERR_ARG, "launch: list_cap above 8192");
  int rc = ensure_outputs(c, m, list_cap);
  if (rc != ABYSS_OK) return rc;
  CK(c->lcnt.ensure((size_t)m), "alloc lcnt");
  CK(c->lst.ensure((size_t)m * list_cap), "alloc lst");
  CK(c->part.ensure((size_t)S * m * 6), "alloc part");
  CK(c->items.ensure(1), "alloc items");
  CK(c->ovf_list.ensure((size_t)m), "alloc overflow list");
  CK(cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream), "clear status");
  CK(cudaMemsetAsync(c->ovf.p, 0, sizeof(int), c->stream), "clear ovf");
  CK(cudaMemsetAsync(c->items.p, 0, sizeof(int), c->stream), "clear work queue");
  CK(cudaMemsetAsync(c->lcnt.p, 0, sizeof(int) * (size_t)m, c->stream), "clear list counts");

  JSet js = jset_of(c);
  Work w;
  w.m = m;
  w.n_chunks = S;
  w.chunk_len = L;
  w.cap = list_cap;
  w.eps2 = eps2;
  w.eps2f = (float)eps2;
  w.lcnt = c->lcnt.p;
  w.lst = c->lst.p;
  w.part = c->part.p;
  w.status = c->status.p;
  w.item_counter = c->items.p;
  w.s_stride = S;
  w.items = nullptr;
  w.n_items_dev = nullptr;
  w.m_dev = nullptr;
  w.row_nchunks = nullptr;
  w.row_joff = nullptr;
  w.row_jlen = nullptr;

  if (c->profiling) CK(cudaEventRecord(c->ev[0], c->stream), "event");
  if ((t.kernel == 1 || t.kernel == 3) && t.mode == 1) {
    if (c->cub_bytes == 0 || c->keys.cap < (size_t)m) {
      CK(c->keys.ensure(m), "alloc keys");
      CK(c->keys_alt.ensure(m), "alloc keys");
      CK(c->rows.ensure(m), "alloc rows");
      CK(c->rows_alt.ensure(m), "alloc rows");
      CK(c->bbox.ensure(6), "alloc bbox");
      c->cub_bytes = sort_temp_bytes((int)c->keys.cap);
      CK(c->cub_tmp.ensure(c->cub_bytes), "alloc sort scratch");
    }
    const int per_block = t.threads * t.ipt;
    CK(c->anchor.ensure((size_t)3 * n_iblocks), "alloc anchors");
    launch_spatial_order(c->stream, m, c->targets.p, js, c->bbox.p, c->keys.p, c->keys_alt.p, c->rows.p,
                         c->rows_alt.p, c->cub_tmp.p, c->cub_bytes, c->order_t.p, c->order_o.p, per_block,
                         c->anchor.p, c->sm_count);
    w.order_t = c->order_t.p;
    w.order_o = c->order_o.p;
    w.anchor = c->anchor.p;
  } else {
    w.order_t = c->targets.p;
    w.order_o = c->iota.p;
  }
  if (c->profiling == 1) CK(cudaEventRecord(c->ev[1], c->stream), "event");
  Outputs o;
  o.targets = c->targets.p;
  o.acc_reg = c->acc_reg.p;
  o.jerk_reg = c->jerk_reg.p;
  o.acc_irr = c->acc_irr.p;
  o.jerk_irr = c->jerk_irr.p;
  o.nnb = c->nnb.p;
  o.list = c->list.p;
  o.overflow_rows = c->ovf.p;
  o.ovf_list = c->ovf_list.p;
  if (t.kernel == 4 || t.kernel == 5) {
    if (launch_tile_split(c->stream, t.ipt, t.unroll, t.kernel == 5, grid, js, w, n_iblocks) != 0)
      return fail(c, ABYSS_ERR_ARG, "launch: unsupported tile shape");
    t.grid = grid;
  } else if (t.kernel == 1 || t.kernel == 3) {
    if (launch_tile(c->stream, t.threads, t.ipt, t.mode == 1, t.kernel == 3, t.unroll, t.min_blocks, grid, js,
                    w, n_iblocks) != 0)
      return fail(c, ABYSS_ERR_ARG, "launch: unsupported tile shape");
    t.grid = grid;
  } else {
    // a launch of at most kFuseRows rows finalizes in its force kernel's last block
    if (launch_jmajor(c->stream, t.ipt, js, w, L, m <= kFuseRows ? &o : nullptr) != 0)
      return fail(c, ABYSS_ERR_ARG, "launch: unsupported j-major shape");
  }
  CK(cudaGetLastError(), "force kernel launch");
  if (c->profiling == 1) CK(cudaEventRecord(c->ev[2], c->stream), "event");
  if (!(t.kernel == 2 && m <= kFuseRows)) {
    launch_finalize(c->stream, js, w, o, c->sm_count);
    CK(cudaGetLastError(), "finalize launch");
  }
  if (c->profiling) CK(cudaEventRecord(c->ev[3], c->stream), "event");
  t.j_split = S;
  c->plan = t;
  c->plan_chunks = S;
  c->launched = true;
  c->launched_m = m;
  c->launched_cap = list_cap;
  return ABYSS_OK;
}

int abyss_fetch(abyss_ctx *c, double *acc_reg, double *jerk_reg, double *acc_irr, double *jerk_irr,
                int *nnb, int *list, int *overflow_rows) {
  if (!c) return ABYSS_ERR_ARG;
  if (!c->launched) return fail(c, ABYSS_ERR_STATE, "fetch: nothing launched");
  cudaSetDevice(c->device);
  const size_t m = c->launched_m;
  int st = 0, ovf = 0;
  D2H out;
  CK(out.queue(c, {{&st, c->status.p, sizeof(int)},
                   {&ovf, c->ovf.p, sizeof(int)},
                   {acc_reg, c->acc_reg.p, acc_reg ? m * 24 : 0},
                   {jerk_reg, c->jerk_reg.p, jerk_reg ? m * 24 : 0},
                   {acc_irr, c->acc_irr.p, acc_irr ? m * 24 : 0},
                   {jerk_irr, c->jerk_irr.p, jerk_irr ? m * 24 : 0},
                   {nnb, c->nnb.p, nnb ? m * 4 : 0},
                   {list, c->list.p, list ? m * (size_t)c->launched_cap * 4 : 0}}),
     "D2H results");
  CK(ctx_wait(c), "synchronize");
  out.finish();
  if (overflow_rows) *overflow_rows = ovf;
  if (st & kErrTimeout) return fail(c, ABYSS_ERR_TIMEOUT, "device wait timed out");
  if (ovf > 0) {
    c->err = "neighbour list overflow in " + std::to_string(ovf) + " rows";
    return ABYSS_WARN_OVERFLOW;
  }
  return ABYSS_OK;
}

int abyss_regular_force(abyss_ctx *c, int m, const int *targets, double eps2, int list_cap,
                        const abyss_tuning *tuning, double *acc_reg, double *jerk_reg,
                        double *acc_irr, double *jerk_irr, int *nnb, int *list,
                        int *overflow_rows) {
  int rc = abyss_set_targets(c, m, targets);
  if (rc != ABYSS_OK) return rc;
  rc = abyss_launch(c, eps2, list_cap, tuning);
  if (rc != ABYSS_OK) return rc;
  return abyss_fetch(c, acc_reg, jerk_reg, acc_irr, jerk_irr, nnb, list, overflow_rows);
}

int abyss_tile_variants(void) { return tile_variant_count(); }

int abyss_tile_variant(int i, int *shape6) {
  if (!shape6) return ABYSS_ERR_ARG;
  return tile_variant_shape(i, shape6) == 0 ? ABYSS_OK : ABYSS_ERR_ARG;
}

int abyss_last_plan(const abyss_ctx *c, abyss_tuning *plan, int *n_chunks) {
  if (!c) return ABYSS_ERR_ARG;
  if (plan) *plan = c->plan;
  if (n_chunks) *n_chunks = c->plan_chunks;
  return ABYSS_OK;
}

int abyss_last_order(abyss_ctx *c, int *rows) {
  if (!c || !rows) return ABYSS_ERR_ARG;
  if (!c->launched) return fail(c, ABYSS_ERR_STATE, "last_order: nothing launched");
  cudaSetDevice(c->device);
  const bool ordered = (c->plan.kernel == 1 || c->plan.kernel == 3) && c->plan.mode == 1;
  D2H out;
  CK(out.queue(c, {{rows, ordered ? c->order_o.p : c->iota.p, (size_t)c->launched_m * 4}}), "D2H order");
  CK(ctx_wait(c), "synchronize");
  out.finish();
  return ABYSS_OK;
}

int abyss_set_profiling(abyss_ctx *c, int on) {
  if (!c) return ABYSS_ERR_ARG;
  c->profiling = on == 2 ? 2 : on != 0 ? 1 : 0;
  return ABYSS_OK;
}

int abyss_last_timing(abyss_ctx *c, float *ms3) {
  if (!c || !ms3) return ABYSS_ERR_ARG;
  if (!c->profiling) return fail(c, ABYSS_ERR_STATE, "last_timing: profiling is off");
  cudaSetDevice(c->device);
  CK(ctx_wait(c), "synchronize");
  if (c->profiling == 2) {
    ms3[0] = ms3[2] = 0.0f;
    CK(cudaEventElapsedTime(&ms3[1], c->ev[0], c->ev[3]), "event time");
    return ABYSS_OK;
  }
  for (int i = 0; i < 3; ++i) CK(cudaEventElapsedTime(&ms3[i], c->ev[i], c->ev[i + 1]), "event time");
  return ABYSS_OK;
}

int abyss_set_tuning_table(abyss_ctx *c, int k, const int *m_max, const abyss_tuning *entries) {
  if (!c || k < 0 || (k > 0 && (!m_max || !entries))) return ABYSS_ERR_ARG;
  c->table.m_max.assign(m_max, m_max + k);
  c->table.entries.assign(entries, entries + k);
  return ABYSS_OK;
}

int abyss_energy(abyss_ctx *c, int n, const double *x, const double *v, const double *mass,
                 double eps2, double *energy) {
  if (!c || n <= 0 || !x || !v || !mass || !energy) return fail(c, ABYSS_ERR_ARG, "energy: bad args");
  cudaSetDevice(c->device);
  CK(c->e_x.ensure((size_t)3 * n), "alloc");
  CK(c->e_v.ensure((size_t)3 * n), "alloc");
  CK(c->e_m.ensure(n), "alloc");
  CK(c->e_row.ensure(n), "alloc");
  CK(h2d(c, {{c->e_x.p, x, (size_t)24 * n}, {c->e_v.p, v, (size_t)24 * n}, {c->e_m.p, mass, (size_t)8 * n}}),
     "H2D");
  launch_energy(c->stream, n, c->e_x.p, c->e_v.p, c->e_m.p, eps2, c->e_row.p);
  CK(cudaGetLastError(), "energy launch");
  std::vector<double> rows(n);
  D2H out;
  CK(out.queue(c, {{rows.data(), c->e_row.p, (size_t)8 * n}}), "D2H");
  CK(ctx_wait(c), "synchronize");
  out.finish();
  double e = 0.0;
  for (int i = 0; i < n; ++i) e += rows[i];
  *energy = e;
  return ABYSS_OK;
}

int abyss_init_derivs23(abyss_ctx *c, int n, const double *x, const double *v, const double *mass,
                        const double *r2nb, const double *a0, const double *a1, double eps2,
                        double *reg2, double *reg3, double *irr2, double *irr3) {
  if (!c || n <= 0 || !x || !v || !mass || !r2nb || !a0 || !a1 || !reg2 || !reg3 || !irr2 || !irr3)
    return fail(c, ABYSS_ERR_ARG, "init_derivs23: bad args");
  if (!(eps2 >= 0.0)) return fail(c, ABYSS_ERR_ARG, "init_derivs23: eps2 must be >= 0");
  cudaSetDevice(c->device);
  const size_t n3 = (size_t)3 * n;
  CK(c->e_x.ensure(n3), "alloc");
  CK(c->e_v.ensure(n3), "alloc");
  CK(c->e_m.ensure(n), "alloc");
  CK(c->i_a0.ensure(n3), "alloc");
  CK(c->i_a1.ensure(n3), "alloc");
  CK(c->i_r2.ensure(n), "alloc");
  CK(c->i_out.ensure((size_t)12 * n), "alloc");
  CK(h2d(c, {{c->e_x.p, x, 8 * n3}, {c->e_v.p, v, 8 * n3}, {c->e_m.p, mass, (size_t)8 * n},
             {c->i_a0.p, a0, 8 * n3}, {c->i_a1.p, a1, 8 * n3}, {c->i_r2.p, r2nb, (size_t)8 * n}}),
     "H2D");
  launch_init_derivs23(c->stream, n, c->e_x.p, c->e_v.p, c->i_a0.p, c->i_a1.p, c->e_m.p, c->i_r2.p, eps2,
                       c->i_out.p);
  CK(cudaGetLastError(), "init_derivs23 launch");
  std::vector<double> out((size_t)12 * n);
  D2H res;
  CK(res.queue(c, {{out.data(), c->i_out.p, (size_t)96 * n}}), "D2H");
  CK(ctx_wait(c), "synchronize");
  res.finish();
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      const double *o = &out[(size_t)12 * i];
      reg2[3 * (size_t)i + d] = o[d];
      reg3[3 * (size_t)i + d] = o[3 + d];
      irr2[3 * (size_t)i + d] = o[6 + d];
      irr3[3 * (size_t)i + d] = o[9 + d];
    }
  return ABYSS_OK;
}

}  // extern "C"
