// Regular force for callers that cannot allocate device memory.
//
// Some hosts of this library do not own the GPU's memory: a simulation or ML
// framework that reserves the device through its own caching allocator, a
// process held to a hard device-memory budget, or code on a path where a
// cudaMalloc/cudaFree (which may synchronize the whole device) is not allowed.
// They can still hand over device buffers they already hold for the inputs and
// outputs.  abyss_regular_force_noalloc runs the regular force for them with
// every intermediate buffer (list counters, unsorted lists, chunk partial sums,
// overflowed-row list, the work-queue head and status words) in one fixed array
// of this file,
// g_noalloc_scratch, and calls no allocator at all.
//
// Limits: at most kMaxTargets targets and kMaxCap list entries per target.
// The array lives in every GPU that loads the library until the process exits.
// Calls share it: two calls whose work overlaps on the GPU (different streams,
// or different host threads on one device) race on it, so callers must
// serialize them.  Each call clears what must start at zero and returns only
// after its work has finished.  The first call on a device, with that device
// current, looks up the array's device address (cudaGetSymbolAddress) and fills
// a constant row map.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/abyss_reg.h"
#include "abyss_internal.cuh"
#include "kernels.cuh"

using namespace abyss;

namespace {

constexpr int kMaxTargets = 4096;
constexpr int kMaxCap = 256;
constexpr int kChunks = 8;   // j-chunks per target at most
constexpr int kTJ = 128;     // tile length of the force kernel
constexpr int kMaxDevices = 64;

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kOffIota = 0;
constexpr size_t kOffCnt = kOffIota + align256(sizeof(int) * kMaxTargets);
constexpr size_t kOffLst = kOffCnt + align256(sizeof(int) * kMaxTargets);
constexpr size_t kOffPart = kOffLst + align256(sizeof(int) * (size_t)kMaxTargets * kMaxCap);
constexpr size_t kOffOvf = kOffPart + align256(sizeof(double) * (size_t)kMaxTargets * kChunks * 6);
constexpr size_t kOffCtr = kOffOvf + align256(sizeof(int) * kMaxTargets);
constexpr size_t kScratchBytes = kOffCtr + 256;  // ctr: [0] queue head, [1] status, [2] overflow rows, [3] bad targets

}  // namespace

// The scratch array (about 5.6 MiB).  Host code only ever uses its device
// address from cudaGetSymbolAddress, looked up per device below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

std::mutex g_setup_mu;
unsigned char *g_scratch_addr[kMaxDevices] = {};

__global__ void noalloc_fill_iota(int *out, int m) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) out[i] = i;
}

__global__ void noalloc_check_targets(const int *targets, int m, int n, int *bad) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    if (targets[i] < 0 || targets[i] >= n) atomicAdd(bad, 1);
}

// Device address of the scratch array on the current device (set up once).
int scratch_address(int dev, cudaStream_t s, unsigned char **out) {
  if (dev < 0 || dev >= kMaxDevices) return ABYSS_ERR_NODEVICE;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      std::fprintf(stderr, "abyss_regular_force_noalloc: cudaGetSymbolAddress failed: %s\n",
                   cudaGetErrorString(e));
      return ABYSS_ERR_CUDA;
    }
    unsigned char *base = static_cast<unsigned char *>(p);
    noalloc_fill_iota<<<(kMaxTargets + 255) / 256, 256, 0, s>>>(reinterpret_cast<int *>(base + kOffIota),
                                                                  kMaxTargets);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      std::fprintf(stderr, "abyss_regular_force_noalloc: set-up failed: %s\n", cudaGetErrorString(e));
      return ABYSS_ERR_CUDA;
    }
    g_scratch_addr[dev] = base;
  }
  *out = g_scratch_addr[dev];
  return ABYSS_OK;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int refuse(const char *why) {
  std::fprintf(stderr, "abyss_regular_force_noalloc: %s\n", why);
  return ABYSS_ERR_ARG;
}

}  // namespace

extern "C" int abyss_regular_force_noalloc(int n, const double *px, const double *py, const double *pz,
                                           const float *vm, const double *pvx, const double *pvy,
                                           const double *pvz, const double *mass, const double *r2nb,
                                           int m, const int *targets, double eps2, int list_cap,
                                           double *acc_reg, double *jerk_reg, double *acc_irr,
                                           double *jerk_irr, int *nnb, int *list, void *stream) {
  if (n < 2) return refuse("n must be at least 2");
  if (m <= 0) return refuse("m must be positive");
  if (m > kMaxTargets) {
    std::fprintf(stderr, "abyss_regular_force_noalloc: m = %d exceeds the maximum of %d targets\n", m,
                 kMaxTargets);
    return ABYSS_ERR_ARG;
  }
  if (list_cap <= 0 || list_cap > kMaxCap) {
    std::fprintf(stderr, "abyss_regular_force_noalloc: list_cap = %d outside 1..%d\n", list_cap, kMaxCap);
    return ABYSS_ERR_ARG;
  }
  if (!(eps2 >= 0.0)) return refuse("eps2 must be >= 0");
  const void *in[] = {px, py, pz, vm, pvx, pvy, pvz, mass, r2nb, targets};
  const void *outp[] = {acc_reg, jerk_reg, acc_irr, jerk_irr, nnb, list};
  for (const void *p : in)
    if (!p) return refuse("null input pointer");
  for (const void *p : outp)
    if (!p) return refuse("null output pointer");
  if (!aligned16(px) || !aligned16(py) || !aligned16(pz) || !aligned16(vm))
    return refuse("px, py, pz and vm must be 16-byte aligned device pointers");

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int dev = 0, sm_count = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ABYSS_ERR_NODEVICE;
  if (cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return ABYSS_ERR_CUDA;
  unsigned char *base = nullptr;
  int rc = scratch_address(dev, s, &base);
  if (rc != ABYSS_OK) return rc;
  int *iota = reinterpret_cast<int *>(base + kOffIota);
  int *lcnt = reinterpret_cast<int *>(base + kOffCnt);
  int *lst = reinterpret_cast<int *>(base + kOffLst);
  double *part = reinterpret_cast<double *>(base + kOffPart);
  int *ovf_list = reinterpret_cast<int *>(base + kOffOvf);
  int *ctr = reinterpret_cast<int *>(base + kOffCtr);

  // clear what must start at zero: queue head, status, overflow and bad-target
  // counters, and the list counters of the m rows
  if (cudaMemsetAsync(ctr, 0, 4 * sizeof(int), s) != cudaSuccess ||
      cudaMemsetAsync(lcnt, 0, sizeof(int) * (size_t)m, s) != cudaSuccess)
    return ABYSS_ERR_CUDA;
  // targets live in device memory: check them on the device before any use
  noalloc_check_targets<<<(m + 255) / 256, 256, 0, s>>>(targets, m, n, ctr + 3);
  int host_ctr[4] = {0, 0, 0, 0};
  if (cudaMemcpyAsync(host_ctr, ctr, sizeof(host_ctr), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return ABYSS_ERR_CUDA;
  if (host_ctr[3] != 0) return refuse("a target index is outside 0..n-1");

  // launch shape: packed tile kernel, double-single offsets (no target ordering)
  const int nt = 128, ipt = 2, minb = 4;
  const int occ = tile_occupancy(nt, ipt, false, true, 0, minb);
  if (occ <= 0) return ABYSS_ERR_CUDA;
  const int grid_max = occ * sm_count;
  const int per_block = nt * ipt;
  const int n_iblocks = (m + per_block - 1) / per_block;
  int S = (32 * grid_max + n_iblocks - 1) / n_iblocks;
  S = std::min(S, kChunks);
  S = std::min(S, std::max(1, (n + 2 * kTJ - 1) / (2 * kTJ)));
  S = std::max(S, 1);
  int chunk = ((n + S - 1) / S + kTJ - 1) / kTJ * kTJ;
  S = (n + chunk - 1) / chunk;

  JSet js;
  js.px = px;
  js.py = py;
  js.pz = pz;
  js.vm = reinterpret_cast<const float4 *>(vm);
  js.pvx = pvx;
  js.pvy = pvy;
  js.pvz = pvz;
  js.mass = mass;
  js.r2nb = r2nb;
  js.n = n;
  Work w;
  w.order_t = targets;
  w.order_o = iota;
  w.m = m;
  w.n_chunks = S;
  w.chunk_len = chunk;
  w.cap = list_cap;
  w.eps2 = eps2;
  w.eps2f = (float)eps2;
  w.lcnt = lcnt;
  w.lst = lst;
  w.part = part;
  w.status = ctr + 1;
  w.item_counter = ctr;
  w.s_stride = S;
  w.items = nullptr;
  w.n_items_dev = nullptr;
  w.m_dev = nullptr;
  w.row_nchunks = nullptr;
  w.row_joff = nullptr;
  w.row_jlen = nullptr;
  Outputs o;
  o.targets = targets;
  o.acc_reg = acc_reg;
  o.jerk_reg = jerk_reg;
  o.acc_irr = acc_irr;
  o.jerk_irr = jerk_irr;
  o.nnb = nnb;
  o.list = list;
  o.overflow_rows = ctr + 2;
  o.ovf_list = ovf_list;
  const int grid = std::min(grid_max, n_iblocks * S);
  if (launch_tile(s, nt, ipt, false, true, 0, minb, grid, js, w, n_iblocks) != 0) return ABYSS_ERR_CUDA;
  launch_finalize(s, js, w, o, sm_count);
  if (cudaGetLastError() != cudaSuccess) return ABYSS_ERR_CUDA;
  if (cudaMemcpyAsync(host_ctr, ctr, sizeof(host_ctr), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return ABYSS_ERR_CUDA;
  if (host_ctr[1] & kErrTimeout) return ABYSS_ERR_TIMEOUT;
  return host_ctr[2] > 0 ? ABYSS_WARN_OVERFLOW : ABYSS_OK;
}
