// Batched regular force over an ensemble of independent clusters
// (include/abyss_ens.h).
//
// All clusters live in one set of device arrays (cluster k owns particles
// [off_k, off_k + n_k)).  A wave lists (cluster, targets) blocks; the host turns
// it into a work list of (target slice, j-chunk) items sorted longest first,
// and the device runs
//     predict_multi   every active cluster to its own time
//     reg_force_tile  one persistent launch draining the work list
//     finalize_rows   FP64 sums, sorted cluster-local lists, irregular part
// Counts (rows, items) are read on the device, so the same three kernels can
// be captured once into a CUDA graph and replayed for every wave.
#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/abyss_ens.h"
#include "../../include/abyss_reg.h"
#include "abyss_internal.cuh"
#include "kernels.cuh"

using namespace abyss;

namespace {
constexpr int kSMax = 16;   // j-chunks per cluster at most
constexpr int kTJ = 128;

template <class T>
struct Buf {
  T *p = nullptr;
  size_t n = 0;
  cudaError_t alloc(size_t count) {
    n = std::max<size_t>(count, 1) + kPad;
    return cudaMalloc((void **)&p, n * sizeof(T));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
  }
};
}  // namespace

struct abyss_ens {
  abyss_ctx *ctx = nullptr;
  cudaStream_t stream = nullptr;
  int device = 0, sm_count = 148;
  int nc = 0, n_total = 0, cap = 0;   // nc = cluster slots, n_total = particle capacity
  std::vector<int> n_k, off_k;          // n_k = 0: free slot
  std::map<int, int> free_ranges;       // particle offset -> length, 32-aligned
  long long bytes = 0;
  // state and predicted j-set
  Buf<double> x, v, a0, a1, t0, mass, r2nb, px, py, pz, pvx, pvy, pvz;
  Buf<float4> vm;
  Buf<int> cid, active;
  Buf<double> new_time, scale;
  // wave
  Buf<int> order_t, order_o, row_nch, row_joff, row_jlen, counts;  // counts: [0] rows, [1] items
  Buf<WorkItem> items;
  size_t items_cap = 0;
  // work and outputs
  Buf<int> lcnt, lst, status, ovf, qhead, list, nnb, ovf_list;
  Buf<double> part, acc_reg, jerk_reg, acc_irr, jerk_irr;
  // host wave description
  int rows = 0, n_items = 0, launches = 0;
  std::vector<int> h_order, h_nch, h_joff, h_jlen, h_active;
  std::vector<double> h_time, h_scale;
  std::vector<WorkItem> h_items;
  std::vector<int> wave_clusters, wave_rows_begin, wave_m;
  std::vector<std::vector<WorkItem>> cluster_items;  // plain mode, slices relative to the cluster's rows
  // launch shape
  abyss_tuning shape{};
  int grid = 0;
  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  abyss_tuning graph_shape{};
  double graph_eps2 = -1.0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // pinned host staging of the state arrays, laid out like the device arena
  // (15 doubles per particle: x, v, a0, a1 [3] each, t0, mass, r2nb)
  double *stage = nullptr;
  int chunk_j = 2048;  // j per chunk of a cluster (>= 128): its chunk count is ceil(n_k / chunk_j), <= kSMax
  // tuned chunk lengths by cluster size: the first entry with n_k <= chunk_nmax
  // applies, else chunk_j
  std::vector<int> chunk_nmax, chunk_len;
  // pinned host staging of a wave's description (set_wave) and of its results
  // (fetch_view), so that neither goes through pageable copies
  unsigned char *wstage = nullptr;
  size_t wstage_bytes = 0;
  unsigned char *ostage = nullptr;
  size_t ostage_bytes = 0;
  cudaEvent_t desc_ev = nullptr;  // the wave description's copies out of wstage are done
  bool desc_pending = false;
  // Two waves can be in flight (abyss_ens_submit / abyss_ens_collect): every
  // per-wave buffer above has a twin in `other`, and switching slots swaps
  // them, so the code above always works on the current slot.
  struct Slot *other = nullptr;
  int cur = 0;            // slot number the fields above belong to
  int busy[2] = {0, 0};   // slot s holds a submitted wave not yet collected
  std::string err;
};

// The per-wave state of an ensemble that is not current (see abyss_ens::other).
struct Slot {
  Buf<int> active, order_t, row_nch, row_joff, row_jlen, counts, lcnt, lst, status, ovf, qhead, list, nnb, ovf_list;
  Buf<WorkItem> items;
  Buf<double> new_time, scale, part, acc_reg, jerk_reg, acc_irr, jerk_irr;
  int rows = 0, n_items = 0, launches = 0;
  std::vector<int> h_order, h_nch, h_joff, h_jlen, h_active;
  std::vector<double> h_time, h_scale;
  std::vector<WorkItem> h_items;
  std::vector<int> wave_clusters, wave_rows_begin, wave_m;
  std::vector<std::vector<WorkItem>> cluster_items;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  abyss_tuning graph_shape{};
  double graph_eps2 = -1.0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, desc_ev = nullptr;
  bool desc_pending = false;
  unsigned char *wstage = nullptr, *ostage = nullptr;
  size_t wstage_bytes = 0, ostage_bytes = 0;
};

namespace {

int efail(abyss_ens *e, int code, const std::string &m) {
  if (e) e->err = m;
  return code;
}

// Make the other slot current (its buffers must exist: abyss_ens_pipeline).
void swap_slot(abyss_ens *e) {
  Slot &o = *e->other;
  std::swap(e->active, o.active);
  std::swap(e->order_t, o.order_t);
  std::swap(e->row_nch, o.row_nch);
  std::swap(e->row_joff, o.row_joff);
  std::swap(e->row_jlen, o.row_jlen);
  std::swap(e->counts, o.counts);
  std::swap(e->items, o.items);
  std::swap(e->lcnt, o.lcnt);
  std::swap(e->lst, o.lst);
  std::swap(e->status, o.status);
  std::swap(e->ovf, o.ovf);
  std::swap(e->qhead, o.qhead);
  std::swap(e->list, o.list);
  std::swap(e->nnb, o.nnb);
  std::swap(e->ovf_list, o.ovf_list);
  std::swap(e->new_time, o.new_time);
  std::swap(e->scale, o.scale);
  std::swap(e->part, o.part);
  std::swap(e->acc_reg, o.acc_reg);
  std::swap(e->jerk_reg, o.jerk_reg);
  std::swap(e->acc_irr, o.acc_irr);
  std::swap(e->jerk_irr, o.jerk_irr);
  std::swap(e->rows, o.rows);
  std::swap(e->n_items, o.n_items);
  std::swap(e->launches, o.launches);
  std::swap(e->h_order, o.h_order);
  std::swap(e->h_nch, o.h_nch);
  std::swap(e->h_joff, o.h_joff);
  std::swap(e->h_jlen, o.h_jlen);
  std::swap(e->h_active, o.h_active);
  std::swap(e->h_time, o.h_time);
  std::swap(e->h_scale, o.h_scale);
  std::swap(e->h_items, o.h_items);
  std::swap(e->wave_clusters, o.wave_clusters);
  std::swap(e->wave_rows_begin, o.wave_rows_begin);
  std::swap(e->wave_m, o.wave_m);
  std::swap(e->cluster_items, o.cluster_items);
  std::swap(e->graph, o.graph);
  std::swap(e->graph_exec, o.graph_exec);
  std::swap(e->graph_shape, o.graph_shape);
  std::swap(e->graph_eps2, o.graph_eps2);
  std::swap(e->ev0, o.ev0);
  std::swap(e->ev1, o.ev1);
  std::swap(e->desc_ev, o.desc_ev);
  std::swap(e->desc_pending, o.desc_pending);
  std::swap(e->wstage, o.wstage);
  std::swap(e->ostage, o.ostage);
  std::swap(e->wstage_bytes, o.wstage_bytes);
  std::swap(e->ostage_bytes, o.ostage_bytes);
  e->cur ^= 1;
}

#define ECK(expr, what)                                                                          \
  do {                                                                                           \
    cudaError_t _e = (expr);                                                                     \
    if (_e != cudaSuccess)                                                                       \
      return efail(e, _e == cudaErrorMemoryAllocation ? ABYSS_ERR_OOM : ABYSS_ERR_CUDA,          \
                   std::string(what) + ": " + cudaGetErrorString(_e));                           \
  } while (0)

JSet jset_of(abyss_ens *e) {
  JSet js;
  js.px = e->px.p;
  js.py = e->py.p;
  js.pz = e->pz.p;
  js.vm = e->vm.p;
  js.pvx = e->pvx.p;
  js.pvy = e->pvy.p;
  js.pvz = e->pvz.p;
  js.mass = e->mass.p;
  js.r2nb = e->r2nb.p;
  js.n = e->n_total;
  return js;
}

// Work and outputs of the batched wave (device counts) or of one cluster
// (plain mode: row and item pointers offset to the cluster's slice).
void make_work(abyss_ens *e, double eps2, int row_begin, const WorkItem *items, const int *n_items_dev,
               const int *m_dev, int m_host, Work &w, Outputs &o) {
  w.order_t = e->order_t.p + row_begin;
  w.order_o = e->order_o.p;  // identity rows; slices index from 0
  w.m = m_host;
  w.n_chunks = kSMax;
  w.chunk_len = 0;
  w.cap = e->cap;
  w.eps2 = eps2;
  w.eps2f = (float)eps2;
  w.lcnt = e->lcnt.p + row_begin;
  w.lst = e->lst.p + (size_t)row_begin * e->cap;
  w.part = e->part.p + (size_t)row_begin * kSMax * 6;
  w.status = e->status.p;
  w.item_counter = e->qhead.p;
  w.s_stride = kSMax;
  w.items = items;
  w.n_items_dev = n_items_dev;
  w.m_dev = m_dev;
  w.row_nchunks = e->row_nch.p + row_begin;
  w.row_joff = e->row_joff.p + row_begin;
  w.row_jlen = e->row_jlen.p + row_begin;
  o.targets = e->order_t.p + row_begin;
  o.acc_reg = e->acc_reg.p + 3 * (size_t)row_begin;
  o.jerk_reg = e->jerk_reg.p + 3 * (size_t)row_begin;
  o.acc_irr = e->acc_irr.p + 3 * (size_t)row_begin;
  o.jerk_irr = e->jerk_irr.p + 3 * (size_t)row_begin;
  o.nnb = e->nnb.p + row_begin;
  o.list = e->list.p + (size_t)row_begin * e->cap;
  o.overflow_rows = e->ovf.p;
  o.ovf_list = e->ovf_list.p + row_begin;
}

// The batched wave: reset, predict, one tile launch, finalize.  Everything
// depends only on device memory and fixed pointers, so it can be captured.
int enqueue_batched(abyss_ens *e, double eps2) {
  cudaStream_t s = e->stream;
  ECK(cudaMemsetAsync(e->qhead.p, 0, sizeof(int), s), "reset queue");
  ECK(cudaMemsetAsync(e->status.p, 0, sizeof(int), s), "reset status");
  ECK(cudaMemsetAsync(e->ovf.p, 0, sizeof(int), s), "reset overflow");
  ECK(cudaMemsetAsync(e->lcnt.p, 0, sizeof(int) * (size_t)e->n_total, s), "reset list counts");
  launch_predict_multi(s, e->n_total, e->cid.p, e->active.p, e->new_time.p, e->scale.p, e->x.p, e->v.p,
                       e->a0.p, e->a1.p, e->t0.p, e->mass.p, e->px.p, e->py.p, e->pz.p, e->pvx.p,
                       e->pvy.p, e->pvz.p, e->vm.p, e->sm_count);
  JSet js = jset_of(e);
  Work w;
  Outputs o;
  make_work(e, eps2, 0, e->items.p, e->counts.p + 1, e->counts.p, e->n_total, w, o);
  if (launch_tile(s, e->shape.threads, e->shape.ipt, e->shape.mode == 1, e->shape.kernel == 3, e->shape.unroll,
                  e->shape.min_blocks, e->grid, js, w, 0) != 0)
    return efail(e, ABYSS_ERR_ARG, "unsupported tile shape");
  launch_finalize_grid(s, js, w, o, e->sm_count * 32);
  ECK(cudaGetLastError(), "batched wave launch");
  return ABYSS_OK;
}

}  // namespace

extern "C" {

int abyss_ens_create_arena(abyss_ctx *ctx, int capacity, int max_clusters, int list_cap, abyss_ens **out) {
  if (!ctx || capacity < 2 || max_clusters <= 0 || list_cap <= 0 || list_cap > 8192 || !out) return ABYSS_ERR_ARG;
  abyss_ens *e = new abyss_ens;
  e->ctx = ctx;
  e->stream = ctx_stream(ctx);
  e->device = ctx_device(ctx);
  e->sm_count = ctx_sm_count(ctx);
  cudaSetDevice(e->device);
  e->nc = max_clusters;
  e->cap = list_cap;
  e->n_total = (capacity + 31) / 32 * 32;
  e->n_k.assign(max_clusters, 0);
  e->off_k.assign(max_clusters, 0);
  e->free_ranges[0] = e->n_total;
  const size_t n = e->n_total;
  e->shape.kernel = 3;
  e->shape.mode = 2;
  e->shape.threads = 128;
  e->shape.ipt = 2;
  e->shape.min_blocks = 4;
  e->items_cap = ((size_t)n / 128 + (size_t)max_clusters) * kSMax;
  cudaError_t err = cudaSuccess;
  auto A = [&](auto &b, size_t count) {
    if (err == cudaSuccess) {
      err = b.alloc(count);
      e->bytes += (long long)b.n * (long long)sizeof(*b.p);
    }
  };
  A(e->x, 3 * n); A(e->v, 3 * n); A(e->a0, 3 * n); A(e->a1, 3 * n);
  A(e->t0, n); A(e->mass, n + 2); A(e->r2nb, n + 2);
  A(e->px, n + 2); A(e->py, n + 2); A(e->pz, n + 2); A(e->pvx, n + 2); A(e->pvy, n + 2); A(e->pvz, n + 2);
  A(e->vm, n + 2); A(e->cid, n); A(e->active, max_clusters); A(e->new_time, max_clusters); A(e->scale, max_clusters);
  A(e->order_t, n); A(e->order_o, n); A(e->row_nch, n); A(e->row_joff, n); A(e->row_jlen, n); A(e->counts, 2);
  A(e->ovf_list, n);
  A(e->items, 2 * e->items_cap);  // the batched list, then per-cluster lists of the plain mode
  A(e->lcnt, n); A(e->lst, n * (size_t)list_cap); A(e->status, 1); A(e->ovf, 1); A(e->qhead, 1);
  A(e->list, n * (size_t)list_cap); A(e->nnb, n);
  A(e->part, n * (size_t)kSMax * 6);
  A(e->acc_reg, 3 * n); A(e->jerk_reg, 3 * n); A(e->acc_irr, 3 * n); A(e->jerk_irr, 3 * n);
  if (err == cudaSuccess) err = cudaEventCreate(&e->ev0);
  if (err == cudaSuccess) err = cudaEventCreate(&e->ev1);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->desc_ev, cudaEventDisableTiming);
  if (err != cudaSuccess) {
    abyss_ens_destroy(e);
    return err == cudaErrorMemoryAllocation ? ABYSS_ERR_OOM : ABYSS_ERR_CUDA;
  }
  // every particle slot starts unowned (cluster id -1), rows map to themselves
  std::vector<int> iota(n);
  std::iota(iota.begin(), iota.end(), 0);
  cudaMemset(e->cid.p, 0xff, n * sizeof(int));
  cudaMemcpy(e->order_o.p, iota.data(), n * 4, cudaMemcpyHostToDevice);
  cudaMemset(e->active.p, 0, sizeof(int) * max_clusters);
  e->h_active.assign(max_clusters, 0);
  e->h_time.assign(max_clusters, 0.0);
  e->h_scale.assign(max_clusters, 1.0);
  const int occ = tile_occupancy(e->shape.threads, e->shape.ipt, e->shape.mode == 1, e->shape.kernel == 3,
                                 e->shape.unroll, e->shape.min_blocks);
  e->grid = std::max(1, occ) * e->sm_count;
  if (cudaDeviceSynchronize() != cudaSuccess) {
    abyss_ens_destroy(e);
    return ABYSS_ERR_CUDA;
  }
  *out = e;
  return ABYSS_OK;
}

int abyss_ens_attach(abyss_ens *e, int n, int *k_out) {
  if (!e || n < 2 || !k_out) return ABYSS_ERR_ARG;
  cudaSetDevice(e->device);
  int k = -1;
  for (int i = 0; i < e->nc; ++i)
    if (e->n_k[i] == 0) {
      k = i;
      break;
    }
  if (k < 0) return efail(e, ABYSS_ERR_OOM, "attach: no free cluster slot");
  // Every cluster starts on a 32-particle boundary: the force kernel's TMA bulk
  // copies need 16-byte aligned sources (an even index for the FP64 arrays).
  const int len = (n + 31) / 32 * 32;
  auto it = e->free_ranges.begin();
  for (; it != e->free_ranges.end(); ++it)
    if (it->second >= len) break;
  if (it == e->free_ranges.end()) return efail(e, ABYSS_ERR_OOM, "attach: no room for the cluster");
  const int off = it->first, rest = it->second - len;
  e->free_ranges.erase(it);
  if (rest > 0) e->free_ranges[off + len] = rest;
  std::vector<int> cid(len, -1);
  std::fill(cid.begin(), cid.begin() + n, k);
  ECK(cudaMemcpyAsync(e->cid.p + off, cid.data(), 4 * (size_t)len, cudaMemcpyHostToDevice, e->stream), "H2D cid");
  ECK(cudaStreamSynchronize(e->stream), "attach");
  e->n_k[k] = n;
  e->off_k[k] = off;
  *k_out = k;
  return ABYSS_OK;
}

int abyss_ens_detach(abyss_ens *e, int k) {
  if (!e || k < 0 || k >= e->nc || e->n_k[k] == 0) return ABYSS_ERR_ARG;
  cudaSetDevice(e->device);
  const int off = e->off_k[k], len = (e->n_k[k] + 31) / 32 * 32;
  ECK(cudaMemsetAsync(e->cid.p + off, 0xff, 4 * (size_t)len, e->stream), "clear cid");
  ECK(cudaStreamSynchronize(e->stream), "detach");
  e->n_k[k] = 0;
  e->h_active[k] = 0;
  // return the range and merge it with free neighbours
  auto it = e->free_ranges.emplace(off, len).first;
  auto nx = std::next(it);
  if (nx != e->free_ranges.end() && it->first + it->second == nx->first) {
    it->second += nx->second;
    e->free_ranges.erase(nx);
  }
  if (it != e->free_ranges.begin()) {
    auto pv = std::prev(it);
    if (pv->first + pv->second == it->first) {
      pv->second += it->second;
      e->free_ranges.erase(it);
    }
  }
  return ABYSS_OK;
}

int abyss_ens_free_particles(const abyss_ens *e) {
  if (!e) return ABYSS_ERR_ARG;
  int best = 0;
  for (const auto &r : e->free_ranges) best = std::max(best, r.second);
  return best;
}

int abyss_ens_create(abyss_ctx *ctx, int n_clusters, const int *n_per_cluster, int list_cap,
                     abyss_ens **out) {
  if (!ctx || n_clusters <= 0 || !n_per_cluster || list_cap <= 0 || list_cap > 8192 || !out)
    return ABYSS_ERR_ARG;
  long long tot = 0;
  for (int k = 0; k < n_clusters; ++k) {
    if (n_per_cluster[k] < 2) return ABYSS_ERR_ARG;
    tot += (n_per_cluster[k] + 31) / 32 * 32;
  }
  if (tot > (1ll << 30)) return ABYSS_ERR_ARG;
  abyss_ens *e = nullptr;
  int rc = abyss_ens_create_arena(ctx, (int)tot, n_clusters, list_cap, &e);
  if (rc != ABYSS_OK) return rc;
  for (int k = 0; k < n_clusters; ++k) {
    int slot = -1;
    rc = abyss_ens_attach(e, n_per_cluster[k], &slot);
    if (rc != ABYSS_OK || slot != k) {
      abyss_ens_destroy(e);
      return rc != ABYSS_OK ? rc : ABYSS_ERR_STATE;
    }
  }
  *out = e;
  return ABYSS_OK;
}

int abyss_ens_destroy(abyss_ens *e) {
  if (!e) return ABYSS_ERR_ARG;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
  if (e->graph) cudaGraphDestroy(e->graph);
  Buf<double> *d[] = {&e->x, &e->v, &e->a0, &e->a1, &e->t0, &e->mass, &e->r2nb, &e->px, &e->py, &e->pz,
                      &e->pvx, &e->pvy, &e->pvz, &e->new_time, &e->scale, &e->part, &e->acc_reg,
                      &e->jerk_reg, &e->acc_irr, &e->jerk_irr};
  for (auto *b : d) b->release();
  Buf<int> *i[] = {&e->cid, &e->active, &e->order_t, &e->order_o, &e->row_nch, &e->row_joff, &e->row_jlen,
                   &e->ovf_list, &e->counts,
                   &e->lcnt, &e->lst, &e->status, &e->ovf, &e->qhead, &e->list, &e->nnb};
  for (auto *b : i) b->release();
  e->vm.release();
  e->items.release();
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  if (e->stage) cudaFreeHost(e->stage);
  if (e->wstage) cudaFreeHost(e->wstage);
  if (e->ostage) cudaFreeHost(e->ostage);
  if (e->desc_ev) cudaEventDestroy(e->desc_ev);
  if (e->other) {
    Slot &o = *e->other;
    Buf<int> *bi[] = {&o.active, &o.order_t, &o.row_nch, &o.row_joff, &o.row_jlen, &o.counts, &o.lcnt,
                      &o.lst, &o.status, &o.ovf, &o.qhead, &o.list, &o.nnb, &o.ovf_list};
    for (auto *b : bi) b->release();
    o.items.release();
    Buf<double> *bd[] = {&o.new_time, &o.scale, &o.part, &o.acc_reg, &o.jerk_reg, &o.acc_irr, &o.jerk_irr};
    for (auto *b : bd) b->release();
    if (o.graph_exec) cudaGraphExecDestroy(o.graph_exec);
    if (o.graph) cudaGraphDestroy(o.graph);
    cudaEvent_t ev[] = {o.ev0, o.ev1, o.desc_ev};
    for (auto v : ev)
      if (v) cudaEventDestroy(v);
    if (o.wstage) cudaFreeHost(o.wstage);
    if (o.ostage) cudaFreeHost(o.ostage);
    delete e->other;
  }
  delete e;
  return ABYSS_OK;
}

long long abyss_ens_device_bytes(const abyss_ens *e) { return e ? e->bytes : 0; }

int abyss_ens_list_cap(const abyss_ens *e) { return e ? e->cap : 0; }

int abyss_ens_set_chunk(abyss_ens *e, int j_per_chunk) {
  if (!e || j_per_chunk < kTJ) return ABYSS_ERR_ARG;
  e->chunk_j = j_per_chunk;
  return ABYSS_OK;
}

int abyss_ens_set_tuning(abyss_ens *e, const abyss_tuning *shape, int k, const int *n_max,
                         const int *j_per_chunk) {
  if (!e || k < 0 || (k > 0 && (!n_max || !j_per_chunk))) return ABYSS_ERR_ARG;
  for (int q = 0; q < k; ++q)
    if (j_per_chunk[q] < kTJ || n_max[q] <= 0 || (q > 0 && n_max[q] <= n_max[q - 1]))
      return efail(e, ABYSS_ERR_ARG, "set_tuning: chunk table must rise in n_max, chunks >= 128 j");
  if (e->busy[0] || e->busy[1]) return efail(e, ABYSS_ERR_STATE, "set_tuning: a submitted wave is not collected yet");
  if (shape) {
    abyss_tuning t = *shape;
    if (t.kernel != 1 && t.kernel != 3) return efail(e, ABYSS_ERR_ARG, "set_tuning: ensemble needs a tile kernel");
    if (t.mode == 0) t.mode = 2;
    // a wave's clusters are not spatially ordered: anchor offsets would be inaccurate
    if (t.mode != 2) return efail(e, ABYSS_ERR_ARG, "set_tuning: ensemble needs double-single offsets");
    if (t.threads == 0) t.threads = 128;
    if (t.ipt == 0) t.ipt = t.kernel == 3 ? 2 : 1;
    // the work-list capacity assumes at least 128 targets per block
    if (t.threads * t.ipt < 128) return efail(e, ABYSS_ERR_ARG, "set_tuning: fewer than 128 targets per block");
    const int occ = tile_occupancy(t.threads, t.ipt, false, t.kernel == 3, t.unroll, t.min_blocks);
    if (occ <= 0) return efail(e, ABYSS_ERR_ARG, "set_tuning: not a compiled tile shape");
    t.j_split = 0;
    t.grid = 0;
    e->shape = t;
    e->grid = occ * e->sm_count;
  }
  e->chunk_nmax.assign(n_max, n_max + k);
  e->chunk_len.assign(j_per_chunk, j_per_chunk + k);
  e->rows = 0;  // the next wave is laid out with the new shape
  return ABYSS_OK;
}

int abyss_ens_get_shape(const abyss_ens *e, abyss_tuning *shape) {
  if (!e || !shape) return ABYSS_ERR_ARG;
  *shape = e->shape;
  return ABYSS_OK;
}

int abyss_ens_stage(abyss_ens *e, int k, double **x, double **v, double **a0, double **a1, double **t0,
                    double **mass, double **r2nb) {
  if (!e || k < 0 || k >= e->nc || e->n_k[k] == 0 || !x || !v || !a0 || !a1 || !t0 || !mass || !r2nb)
    return ABYSS_ERR_ARG;
  if (!e->stage) return efail(e, ABYSS_ERR_STATE, "stage: call abyss_ens_stage_reserve first");
  const size_t N = (size_t)e->n_total, off = e->off_k[k];
  double *b = e->stage;
  *x = b + 3 * off;
  *v = b + 3 * N + 3 * off;
  *a0 = b + 6 * N + 3 * off;
  *a1 = b + 9 * N + 3 * off;
  *t0 = b + 12 * N + off;
  *mass = b + 13 * N + off;
  *r2nb = b + 14 * N + off;
  return ABYSS_OK;
}

int abyss_ens_stage_reserve(abyss_ens *e) {
  if (!e) return ABYSS_ERR_ARG;
  if (e->stage) return ABYSS_OK;
  cudaSetDevice(e->device);
  ECK(cudaMallocHost((void **)&e->stage, (size_t)15 * e->n_total * sizeof(double)), "pinned staging");
  return ABYSS_OK;
}

int abyss_ens_upload_staged(abyss_ens *e, int nk, const int *clusters) {
  if (!e || nk < 0 || (nk > 0 && !clusters)) return ABYSS_ERR_ARG;
  if (!e->stage) return efail(e, ABYSS_ERR_STATE, "upload_staged: nothing staged");
  if (nk == 0) return ABYSS_OK;
  std::vector<char> listed(e->nc, 0);
  for (int i = 0; i < nk; ++i) {
    const int k = clusters[i];
    if (k < 0 || k >= e->nc || e->n_k[k] == 0) return efail(e, ABYSS_ERR_ARG, "upload_staged: bad cluster");
    listed[k] = 1;
  }
  // walk every placed cluster in arena order; a run of listed clusters is copied
  // in one go (free gaps inside it are copied too), and an unlisted cluster ends
  // the run, so its device state is never touched
  std::vector<std::pair<int, int>> placed;  // (offset, cluster)
  for (int k = 0; k < e->nc; ++k)
    if (e->n_k[k] > 0) placed.emplace_back(e->off_k[k], k);
  std::sort(placed.begin(), placed.end());
  cudaSetDevice(e->device);
  cudaStream_t s = e->stream;
  const size_t N = (size_t)e->n_total;
  const double *b = e->stage;
  auto copy = [&](size_t lo, size_t hi) -> int {
    const size_t n = hi - lo;
    ECK(cudaMemcpyAsync(e->x.p + 3 * lo, b + 3 * lo, 24 * n, cudaMemcpyHostToDevice, s), "H2D x");
    ECK(cudaMemcpyAsync(e->v.p + 3 * lo, b + 3 * N + 3 * lo, 24 * n, cudaMemcpyHostToDevice, s), "H2D v");
    ECK(cudaMemcpyAsync(e->a0.p + 3 * lo, b + 6 * N + 3 * lo, 24 * n, cudaMemcpyHostToDevice, s), "H2D a0");
    ECK(cudaMemcpyAsync(e->a1.p + 3 * lo, b + 9 * N + 3 * lo, 24 * n, cudaMemcpyHostToDevice, s), "H2D a1");
    ECK(cudaMemcpyAsync(e->t0.p + lo, b + 12 * N + lo, 8 * n, cudaMemcpyHostToDevice, s), "H2D t0");
    ECK(cudaMemcpyAsync(e->mass.p + lo, b + 13 * N + lo, 8 * n, cudaMemcpyHostToDevice, s), "H2D mass");
    ECK(cudaMemcpyAsync(e->r2nb.p + lo, b + 14 * N + lo, 8 * n, cudaMemcpyHostToDevice, s), "H2D r2nb");
    return ABYSS_OK;
  };
  bool open = false;
  size_t lo = 0, hi = 0;
  for (const auto &pk : placed) {
    const int k = pk.second;
    if (listed[k]) {
      if (!open) {
        lo = (size_t)e->off_k[k];
        open = true;
      }
      hi = (size_t)e->off_k[k] + e->n_k[k];
    } else if (open) {
      const int rc = copy(lo, hi);
      if (rc != ABYSS_OK) return rc;
      open = false;
    }
  }
  if (open) return copy(lo, hi);
  return ABYSS_OK;
}

int abyss_ens_upload_state(abyss_ens *e, int k, const double *x, const double *v, const double *a0,
                           const double *a1, const double *t0, const double *mass, const double *r2nb) {
  if (!e || k < 0 || k >= e->nc || e->n_k[k] == 0 || !x || !v || !a0 || !a1 || !t0 || !mass || !r2nb)
    return ABYSS_ERR_ARG;
  cudaSetDevice(e->device);
  const size_t off = e->off_k[k], n = e->n_k[k];
  cudaStream_t s = e->stream;
  ECK(cudaMemcpyAsync(e->x.p + 3 * off, x, 24 * n, cudaMemcpyHostToDevice, s), "H2D x");
  ECK(cudaMemcpyAsync(e->v.p + 3 * off, v, 24 * n, cudaMemcpyHostToDevice, s), "H2D v");
  ECK(cudaMemcpyAsync(e->a0.p + 3 * off, a0, 24 * n, cudaMemcpyHostToDevice, s), "H2D a0");
  ECK(cudaMemcpyAsync(e->a1.p + 3 * off, a1, 24 * n, cudaMemcpyHostToDevice, s), "H2D a1");
  ECK(cudaMemcpyAsync(e->t0.p + off, t0, 8 * n, cudaMemcpyHostToDevice, s), "H2D t0");
  ECK(cudaMemcpyAsync(e->mass.p + off, mass, 8 * n, cudaMemcpyHostToDevice, s), "H2D mass");
  ECK(cudaMemcpyAsync(e->r2nb.p + off, r2nb, 8 * n, cudaMemcpyHostToDevice, s), "H2D r2nb");
  ECK(cudaStreamSynchronize(s), "upload");
  return ABYSS_OK;
}

int abyss_ens_set_wave(abyss_ens *e, int nk, const int *clusters, const double *new_time,
                       const double *time_scale, const int *m_per, const int *targets_local) {
  if (!e || nk <= 0 || !clusters || !new_time || !time_scale || !m_per || !targets_local)
    return efail(e, ABYSS_ERR_ARG, "set_wave: bad arguments");
  if (e->busy[e->cur]) return efail(e, ABYSS_ERR_STATE, "set_wave: a submitted wave is not collected yet");
  cudaSetDevice(e->device);
  std::vector<char> seen(e->nc, 0);
  const int per_block = e->shape.threads * e->shape.ipt;
  e->h_order.clear();
  e->h_nch.clear();
  e->h_joff.clear();
  e->h_jlen.clear();
  e->h_items.clear();
  e->wave_clusters.assign(clusters, clusters + nk);
  e->wave_rows_begin.assign(nk, 0);
  e->wave_m.assign(m_per, m_per + nk);
  e->cluster_items.assign(nk, {});
  std::fill(e->h_active.begin(), e->h_active.end(), 0);
  // A cluster's j-chunking depends on its own size only (chunks of at least
  // chunk_j particles, at most kSMax of them), so its rows are summed in the
  // same order whatever else is in the wave: a cluster's result is the same
  // alone and in any mix, bit for bit.
  const int *tp = targets_local;
  int row = 0;
  for (int i = 0; i < nk; ++i) {
    const int k = clusters[i];
    if (k < 0 || k >= e->nc || e->n_k[k] == 0 || seen[k])
      return efail(e, ABYSS_ERR_ARG, "set_wave: bad, detached or repeated cluster");
    seen[k] = 1;
    const int m = m_per[i], nkp = e->n_k[k], off = e->off_k[k];
    if (m <= 0 || m > nkp) return efail(e, ABYSS_ERR_ARG, "set_wave: bad target count");
    e->h_active[k] = 1;
    e->h_time[k] = new_time[i];
    e->h_scale[k] = time_scale[i];
    int cj = e->chunk_j;
    for (size_t q = 0; q < e->chunk_nmax.size(); ++q)
      if (nkp <= e->chunk_nmax[q]) {
        cj = e->chunk_len[q];
        break;
      }
    int S = std::max(1, std::min(kSMax, (nkp + cj - 1) / cj));
    int chunk = ((nkp + S - 1) / S + kTJ - 1) / kTJ * kTJ;
    S = (nkp + chunk - 1) / chunk;
    e->wave_rows_begin[i] = row;
    for (int q = 0; q < m; ++q) {
      const int t = tp[q];
      if (t < 0 || t >= nkp) return efail(e, ABYSS_ERR_ARG, "set_wave: target index out of range");
      e->h_order.push_back(off + t);
      e->h_nch.push_back(S);
      e->h_joff.push_back(off);
      e->h_jlen.push_back(nkp);
    }
    for (int b = 0; b < m; b += per_block)
      for (int c = 0; c < S; ++c) {
        WorkItem it{};
        it.t_begin = row + b;
        it.t_count = std::min(per_block, m - b);
        it.j0 = off + c * chunk;
        it.j1 = off + std::min(nkp, (c + 1) * chunk);
        it.ch = c;
        e->h_items.push_back(it);
        WorkItem local = it;
        local.t_begin = b;
        e->cluster_items[i].push_back(local);
      }
    row += m;
    tp += m;
  }
  for (const WorkItem &it : e->h_items)
    if (it.j0 % 2 != 0) return efail(e, ABYSS_ERR_STATE, "set_wave: j-range not 16-byte aligned");
  // longest items first: the work queue then drains evenly
  std::stable_sort(e->h_items.begin(), e->h_items.end(), [](const WorkItem &a, const WorkItem &b) {
    return (long long)a.t_count * (a.j1 - a.j0) > (long long)b.t_count * (b.j1 - b.j0);
  });
  if (e->h_items.size() > e->items_cap) return efail(e, ABYSS_ERR_ARG, "set_wave: too many work items");
  e->rows = row;
  e->n_items = (int)e->h_items.size();
  cudaStream_t s = e->stream;
  // this slot's previous description copies read the pinned staging: let them
  // finish first (a wave of the other slot may still run)
  if (e->desc_pending) ECK(cudaEventSynchronize(e->desc_ev), "set_wave");
  const int counts[2] = {e->rows, e->n_items};
  struct Piece {
    void *dst;
    const void *src;
    size_t bytes;
  };
  const Piece pieces[] = {
      {e->order_t.p, e->h_order.data(), 4 * (size_t)row},
      {e->row_nch.p, e->h_nch.data(), 4 * (size_t)row},
      {e->row_joff.p, e->h_joff.data(), 4 * (size_t)row},
      {e->row_jlen.p, e->h_jlen.data(), 4 * (size_t)row},
      {e->items.p, e->h_items.data(), sizeof(WorkItem) * e->h_items.size()},
      {e->counts.p, counts, sizeof(counts)},
      {e->active.p, e->h_active.data(), 4 * (size_t)e->nc},
      {e->new_time.p, e->h_time.data(), 8 * (size_t)e->nc},
      {e->scale.p, e->h_scale.data(), 8 * (size_t)e->nc},
  };
  size_t total = 0;
  for (const Piece &q : pieces) total += (q.bytes + 15) / 16 * 16;
  if (total > e->wstage_bytes) {
    if (e->wstage) cudaFreeHost(e->wstage);  // its copies are done (desc_ev above)
    e->wstage = nullptr;
    e->wstage_bytes = 0;
    const size_t want = std::max(total, (size_t)1 << 20) * 3 / 2;
    ECK(cudaMallocHost((void **)&e->wstage, want), "pinned wave staging");
    e->wstage_bytes = want;
  }
  size_t at = 0;
  for (const Piece &q : pieces) {
    if (q.bytes) {
      std::memcpy(e->wstage + at, q.src, q.bytes);
      ECK(cudaMemcpyAsync(q.dst, e->wstage + at, q.bytes, cudaMemcpyHostToDevice, s), "H2D wave");
    }
    at += (q.bytes + 15) / 16 * 16;
  }
  ECK(cudaEventRecord(e->desc_ev, s), "event");
  e->desc_pending = true;
  return ABYSS_OK;
}

int abyss_ens_launch(abyss_ens *e, double eps2, int mode, const abyss_tuning *tuning) {
  if (!e || !(eps2 >= 0.0)) return efail(e, ABYSS_ERR_ARG, "launch: bad arguments");
  if (e->rows <= 0) return efail(e, ABYSS_ERR_STATE, "launch: no wave set");
  if (e->busy[e->cur]) return efail(e, ABYSS_ERR_STATE, "launch: a submitted wave is not collected yet");
  cudaSetDevice(e->device);
  cudaStream_t s = e->stream;
  if (tuning && tuning->kernel != 0) {
    abyss_tuning t = *tuning;
    if (t.kernel != 1 && t.kernel != 3) return efail(e, ABYSS_ERR_ARG, "launch: ensemble needs a tile kernel");
    if (t.mode == 0) t.mode = 2;
    if (t.threads == 0) t.threads = 128;
    if (t.ipt == 0) t.ipt = t.kernel == 3 ? 2 : 1;
    if (t.threads * t.ipt != e->shape.threads * e->shape.ipt)
      return efail(e, ABYSS_ERR_ARG, "launch: targets per block must match the wave's work list");
    const int occ = tile_occupancy(t.threads, t.ipt, t.mode == 1, t.kernel == 3, t.unroll, t.min_blocks);
    if (occ <= 0) return efail(e, ABYSS_ERR_ARG, "launch: unsupported tile shape");
    e->shape = t;
    e->grid = occ * e->sm_count;
  }
  ECK(cudaEventRecord(e->ev0, s), "event");
  if (mode == ABYSS_ENS_BATCHED) {
    int rc = enqueue_batched(e, eps2);
    if (rc != ABYSS_OK) return rc;
    e->launches = 3;
  } else if (mode == ABYSS_ENS_GRAPH) {
    const bool same = e->graph_exec && e->graph_eps2 == eps2 &&
                      std::memcmp(&e->graph_shape, &e->shape, sizeof(abyss_tuning)) == 0;
    if (!same) {
      if (e->graph_exec) cudaGraphExecDestroy(e->graph_exec);
      if (e->graph) cudaGraphDestroy(e->graph);
      e->graph_exec = nullptr;
      e->graph = nullptr;
      // attributes are set outside capture
      (void)tile_occupancy(e->shape.threads, e->shape.ipt, e->shape.mode == 1, e->shape.kernel == 3,
                           e->shape.unroll, e->shape.min_blocks);
      ECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
      int rc = enqueue_batched(e, eps2);
      cudaGraph_t g = nullptr;
      cudaError_t ce = cudaStreamEndCapture(s, &g);
      if (rc != ABYSS_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      ECK(ce, "end capture");
      e->graph = g;
      ECK(cudaGraphInstantiate(&e->graph_exec, g, 0), "instantiate graph");
      e->graph_shape = e->shape;
      e->graph_eps2 = eps2;
    }
    ECK(cudaGraphLaunch(e->graph_exec, s), "graph launch");
    e->launches = 3;
  } else if (mode == ABYSS_ENS_PLAIN) {
    // one cluster per launch: predict the cluster, its own work list, its finalize
    ECK(cudaMemsetAsync(e->status.p, 0, sizeof(int), s), "reset status");
    ECK(cudaMemsetAsync(e->ovf.p, 0, sizeof(int), s), "reset overflow");
    ECK(cudaMemsetAsync(e->lcnt.p, 0, sizeof(int) * (size_t)e->rows, s), "reset list counts");
    JSet js = jset_of(e);
    e->launches = 0;
    int ovf_total = 0;
    for (size_t i = 0; i < e->wave_clusters.size(); ++i) {
      const int k = e->wave_clusters[i];
      const int rb = e->wave_rows_begin[i], m = e->wave_m[i];
      const int off = e->off_k[k], nkp = e->n_k[k];
      // the cluster's slice of the ensemble arrays
      launch_predict(s, nkp, e->x.p + 3 * (size_t)off, e->v.p + 3 * (size_t)off, e->a0.p + 3 * (size_t)off,
                     e->a1.p + 3 * (size_t)off, e->t0.p + off, e->mass.p + off, e->h_time[k], e->h_scale[k],
                     e->px.p + off, e->py.p + off, e->pz.p + off, e->pvx.p + off, e->pvy.p + off,
                     e->pvz.p + off, e->vm.p + off, e->sm_count);
      const std::vector<WorkItem> &ci = e->cluster_items[i];
      // per-cluster item list and count after the batched list in device memory
      WorkItem *d_items = e->items.p + e->n_items;
      int *d_cnt = e->counts.p;  // reused per cluster; ordered on the stream
      const int cnts[2] = {m, (int)ci.size()};
      if ((size_t)e->n_items + ci.size() > 2 * e->items_cap)
        return efail(e, ABYSS_ERR_ARG, "launch: work list does not fit");
      ECK(cudaMemcpyAsync(d_items, ci.data(), sizeof(WorkItem) * ci.size(), cudaMemcpyHostToDevice, s),
          "H2D items");
      ECK(cudaMemcpyAsync(d_cnt, cnts, sizeof(cnts), cudaMemcpyHostToDevice, s), "H2D counts");
      ECK(cudaMemsetAsync(e->qhead.p, 0, sizeof(int), s), "reset queue");
      ECK(cudaMemsetAsync(e->ovf.p, 0, sizeof(int), s), "reset overflow");  // per-cluster re-list count
      Work w;
      Outputs o;
      make_work(e, eps2, rb, d_items, d_cnt + 1, d_cnt, m, w, o);
      const int g = std::min(e->grid, (int)ci.size());
      if (launch_tile(s, e->shape.threads, e->shape.ipt, e->shape.mode == 1, e->shape.kernel == 3,
                      e->shape.unroll, e->shape.min_blocks, g, js, w, 0) != 0)
        return efail(e, ABYSS_ERR_ARG, "unsupported tile shape");
      launch_finalize_grid(s, js, w, o, std::max(1, std::min(e->sm_count * 32, (m + 3) / 4)));
      e->launches += 3;
      // the counts buffer is restored for later batched waves
      const int all[2] = {e->rows, e->n_items};
      ECK(cudaMemcpyAsync(d_cnt, all, sizeof(all), cudaMemcpyHostToDevice, s), "H2D counts");
      int ovf_k = 0;
      ECK(cudaMemcpyAsync(&ovf_k, e->ovf.p, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H overflow");
      ECK(cudaStreamSynchronize(s), "plain cluster");  // host arrays reused per cluster
      ovf_total += ovf_k;
    }
    ECK(cudaMemcpyAsync(e->ovf.p, &ovf_total, sizeof(int), cudaMemcpyHostToDevice, s), "H2D overflow");
    ECK(cudaStreamSynchronize(s), "plain wave");
    ECK(cudaGetLastError(), "plain launches");
  } else {
    return efail(e, ABYSS_ERR_ARG, "launch: unknown mode");
  }
  ECK(cudaEventRecord(e->ev1, s), "event");
  return ABYSS_OK;
}

int abyss_ens_fetch_view(abyss_ens *e, const double **acc_reg, const double **jerk_reg, const double **acc_irr,
                         const double **jerk_irr, const int **nnb, const int **list, int *overflow_rows) {
  if (!e || !acc_reg || !jerk_reg || !acc_irr || !jerk_irr || !nnb || !list) return ABYSS_ERR_ARG;
  if (e->busy[e->cur]) return efail(e, ABYSS_ERR_STATE, "fetch: use abyss_ens_collect for a submitted wave");
  cudaSetDevice(e->device);
  cudaStream_t s = e->stream;
  const size_t m = e->rows, cap = (size_t)e->cap;
  const size_t need = 16 + 4 * 24 * m + 4 * m + 4 * m * cap + 64;
  if (need > e->ostage_bytes) {
    ECK(cudaStreamSynchronize(s), "fetch_view");
    if (e->ostage) cudaFreeHost(e->ostage);
    e->ostage = nullptr;
    e->ostage_bytes = 0;
    const size_t want = std::max(need, (size_t)1 << 20) * 3 / 2;
    ECK(cudaMallocHost((void **)&e->ostage, want), "pinned result staging");
    e->ostage_bytes = want;
  }
  unsigned char *b = e->ostage;
  int *st = reinterpret_cast<int *>(b);
  double *d = reinterpret_cast<double *>(b + 16);
  int *nb = reinterpret_cast<int *>(b + 16 + 4 * 24 * m);
  int *ls = nb + m;
  ECK(cudaMemcpyAsync(st, e->status.p, 4, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(st + 1, e->ovf.p, 4, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(d, e->acc_reg.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(d + 3 * m, e->jerk_reg.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(d + 6 * m, e->acc_irr.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(d + 9 * m, e->jerk_irr.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(nb, e->nnb.p, 4 * m, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(ls, e->list.p, 4 * m * cap, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaStreamSynchronize(s), "fetch_view");
  *acc_reg = d;
  *jerk_reg = d + 3 * m;
  *acc_irr = d + 6 * m;
  *jerk_irr = d + 9 * m;
  *nnb = nb;
  *list = ls;
  if (overflow_rows) *overflow_rows = st[1];
  if (st[0] & kErrTimeout) return efail(e, ABYSS_ERR_TIMEOUT, "device wait timed out");
  return st[1] > 0 ? ABYSS_WARN_OVERFLOW : ABYSS_OK;
}

int abyss_ens_pipeline(abyss_ens *e) {
  if (!e) return ABYSS_ERR_ARG;
  if (e->other) return ABYSS_OK;
  cudaSetDevice(e->device);
  e->other = new Slot;
  Slot &o = *e->other;
  const size_t n = e->n_total, nc = e->nc, cap = e->cap;
  cudaError_t err = cudaSuccess;
  auto A = [&](auto &b, size_t count) {
    if (err == cudaSuccess) {
      err = b.alloc(count);
      e->bytes += (long long)b.n * (long long)sizeof(*b.p);
    }
  };
  A(o.active, nc); A(o.new_time, nc); A(o.scale, nc);
  A(o.order_t, n); A(o.row_nch, n); A(o.row_joff, n); A(o.row_jlen, n); A(o.counts, 2);
  A(o.ovf_list, n); A(o.items, 2 * e->items_cap);
  A(o.lcnt, n); A(o.lst, n * cap); A(o.status, 1); A(o.ovf, 1); A(o.qhead, 1);
  A(o.list, n * cap); A(o.nnb, n);
  A(o.part, n * (size_t)kSMax * 6);
  A(o.acc_reg, 3 * n); A(o.jerk_reg, 3 * n); A(o.acc_irr, 3 * n); A(o.jerk_irr, 3 * n);
  if (err == cudaSuccess) err = cudaEventCreate(&o.ev0);
  if (err == cudaSuccess) err = cudaEventCreate(&o.ev1);
  if (err == cudaSuccess) err = cudaEventCreateWithFlags(&o.desc_ev, cudaEventDisableTiming);
  if (err == cudaSuccess) err = cudaMemsetAsync(o.active.p, 0, sizeof(int) * nc, e->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
  o.h_active.assign(nc, 0);
  o.h_time.assign(nc, 0.0);
  o.h_scale.assign(nc, 1.0);
  if (err != cudaSuccess)
    return efail(e, err == cudaErrorMemoryAllocation ? ABYSS_ERR_OOM : ABYSS_ERR_CUDA,
                 std::string("pipeline: ") + cudaGetErrorString(err));
  return ABYSS_OK;
}

int abyss_ens_submit(abyss_ens *e, int nk, const int *clusters, const double *new_time, const double *time_scale,
                     const int *m_per, const int *targets_local, double eps2, int mode, int *ticket) {
  if (!e || !ticket || (mode != ABYSS_ENS_BATCHED && mode != ABYSS_ENS_GRAPH))
    return efail(e, ABYSS_ERR_ARG, "submit: bad arguments");
  int rc = abyss_ens_pipeline(e);
  if (rc != ABYSS_OK) return rc;
  // a free slot: the current one, else the other
  if (e->busy[e->cur]) {
    if (e->busy[e->cur ^ 1]) return efail(e, ABYSS_ERR_STATE, "submit: two waves are in flight already");
    swap_slot(e);
  }
  cudaSetDevice(e->device);
  if ((rc = abyss_ens_upload_staged(e, nk, clusters)) != ABYSS_OK) return rc;
  if ((rc = abyss_ens_set_wave(e, nk, clusters, new_time, time_scale, m_per, targets_local)) != ABYSS_OK) return rc;
  if ((rc = abyss_ens_launch(e, eps2, mode, nullptr)) != ABYSS_OK) return rc;
  // queue the results' copies into this slot's pinned staging behind the wave
  cudaStream_t s = e->stream;
  const size_t m = e->rows, cap = (size_t)e->cap;
  const size_t need = 16 + 4 * 24 * m + 4 * m + 4 * m * cap + 64;
  if (need > e->ostage_bytes) {
    ECK(cudaStreamSynchronize(s), "submit");
    if (e->ostage) cudaFreeHost(e->ostage);
    e->ostage = nullptr;
    e->ostage_bytes = 0;
    const size_t want = std::max(need, (size_t)1 << 20) * 3 / 2;
    ECK(cudaMallocHost((void **)&e->ostage, want), "pinned result staging");
    e->ostage_bytes = want;
  }
  unsigned char *b = e->ostage;
  int *st = reinterpret_cast<int *>(b);
  double *d = reinterpret_cast<double *>(b + 16);
  int *nb = reinterpret_cast<int *>(b + 16 + 4 * 24 * m);
  ECK(cudaMemcpyAsync(st, e->status.p, 4, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(st + 1, e->ovf.p, 4, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(d, e->acc_reg.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(d + 3 * m, e->jerk_reg.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(d + 6 * m, e->acc_irr.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(d + 9 * m, e->jerk_irr.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(nb, e->nnb.p, 4 * m, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(nb + m, e->list.p, 4 * m * cap, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaEventRecord(e->desc_ev, s), "event");  // also marks the result copies
  e->busy[e->cur] = 1;
  *ticket = e->cur;
  return ABYSS_OK;
}

int abyss_ens_ready(abyss_ens *e, int ticket) {
  if (!e || ticket < 0 || ticket > 1 || !e->other || !e->busy[ticket]) return ABYSS_ERR_ARG;
  cudaSetDevice(e->device);
  const cudaEvent_t ev = e->cur == ticket ? e->desc_ev : e->other->desc_ev;
  const cudaError_t q = cudaEventQuery(ev);
  if (q == cudaSuccess) return 1;
  if (q == cudaErrorNotReady) return 0;
  return efail(e, ABYSS_ERR_CUDA, std::string("ready: ") + cudaGetErrorString(q));
}

int abyss_ens_collect(abyss_ens *e, int ticket, const double **acc_reg, const double **jerk_reg,
                      const double **acc_irr, const double **jerk_irr, const int **nnb, const int **list,
                      int *rows, float *gpu_ms) {
  if (!e || ticket < 0 || ticket > 1 || !e->other || !e->busy[ticket] || !acc_reg || !jerk_reg || !acc_irr ||
      !jerk_irr || !nnb || !list || !rows)
    return efail(e, ABYSS_ERR_ARG, "collect: bad ticket or arguments");
  if (e->cur != ticket) swap_slot(e);
  cudaSetDevice(e->device);
  ECK(cudaEventSynchronize(e->desc_ev), "collect");
  e->desc_pending = false;
  e->busy[ticket] = 0;
  const size_t m = e->rows;
  unsigned char *b = e->ostage;
  const int *st = reinterpret_cast<const int *>(b);
  const double *d = reinterpret_cast<const double *>(b + 16);
  const int *nb = reinterpret_cast<const int *>(b + 16 + 4 * 24 * m);
  *acc_reg = d;
  *jerk_reg = d + 3 * m;
  *acc_irr = d + 6 * m;
  *jerk_irr = d + 9 * m;
  *nnb = nb;
  *list = nb + m;
  *rows = (int)m;
  if (gpu_ms) {
    *gpu_ms = 0.0f;
    ECK(cudaEventElapsedTime(gpu_ms, e->ev0, e->ev1), "event time");
  }
  if (st[0] & kErrTimeout) return efail(e, ABYSS_ERR_TIMEOUT, "device wait timed out");
  return st[1] > 0 ? ABYSS_WARN_OVERFLOW : ABYSS_OK;
}

int abyss_ens_fetch(abyss_ens *e, double *acc_reg, double *jerk_reg, double *acc_irr, double *jerk_irr,
                    int *nnb, int *list, int *overflow_rows) {
  if (!e) return ABYSS_ERR_ARG;
  if (e->busy[e->cur]) return efail(e, ABYSS_ERR_STATE, "fetch: use abyss_ens_collect for a submitted wave");
  cudaSetDevice(e->device);
  cudaStream_t s = e->stream;
  const size_t m = e->rows;
  int st = 0, ov = 0;
  ECK(cudaMemcpyAsync(&st, e->status.p, 4, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaMemcpyAsync(&ov, e->ovf.p, 4, cudaMemcpyDeviceToHost, s), "D2H");
  if (acc_reg) ECK(cudaMemcpyAsync(acc_reg, e->acc_reg.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  if (jerk_reg) ECK(cudaMemcpyAsync(jerk_reg, e->jerk_reg.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  if (acc_irr) ECK(cudaMemcpyAsync(acc_irr, e->acc_irr.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  if (jerk_irr) ECK(cudaMemcpyAsync(jerk_irr, e->jerk_irr.p, 24 * m, cudaMemcpyDeviceToHost, s), "D2H");
  if (nnb) ECK(cudaMemcpyAsync(nnb, e->nnb.p, 4 * m, cudaMemcpyDeviceToHost, s), "D2H");
  if (list) ECK(cudaMemcpyAsync(list, e->list.p, 4 * m * e->cap, cudaMemcpyDeviceToHost, s), "D2H");
  ECK(cudaStreamSynchronize(s), "fetch");
  if (overflow_rows) *overflow_rows = ov;
  if (st & kErrTimeout) return efail(e, ABYSS_ERR_TIMEOUT, "device wait timed out");
  return ov > 0 ? ABYSS_WARN_OVERFLOW : ABYSS_OK;
}

int abyss_ens_last_ms(abyss_ens *e, float *ms) {
  if (!e || !ms) return ABYSS_ERR_ARG;
  cudaSetDevice(e->device);
  ECK(cudaEventSynchronize(e->ev1), "event sync");
  ECK(cudaEventElapsedTime(ms, e->ev0, e->ev1), "event time");
  return ABYSS_OK;
}

int abyss_ens_last_stats(const abyss_ens *e, int *rows, int *items, int *launches) {
  if (!e) return ABYSS_ERR_ARG;
  if (rows) *rows = e->rows;
  if (items) *items = e->n_items;
  if (launches) *launches = e->launches;
  return ABYSS_OK;
}

}  // extern "C"
