// Internal device-side layout and helpers of the regular-force library.
//
// HBM layout of one particle set ("j-set") of n particles, all arrays padded to
// a multiple of kPad so that the last bulk-copy tile stays inside the allocation:
//   state   x, v, a0, a1   double [n][3]  (as uploaded, AoS)      -- prediction input
//           t0, mass, r2nb double [n]
//   predicted px, py, pz   double [n]     (SoA, FP64)            -- force-kernel tiles
//           vm             float4 [n]     (vx, vy, vz, m)        -- force-kernel tiles
//           pvx, pvy, pvz  double [n]     (FP64)                 -- exact tests, irregular sums
// Per regular-force call (m targets, S j-chunks, list capacity cap):
//   order_t, order_o int [m]            target particle / output row in processing order
//   lcnt    int    [m]                  neighbours found per target (atomic append)
//   lst     int    [m][cap]             entries in the order found (any chunk order)
//   part    double [m][S][6]            per-chunk regular acc (3) + jerk (3)
//   outputs acc_reg, jerk_reg, acc_irr, jerk_irr double [m][3]; nnb int [m];
//           list int [m][cap]           (final, ascending j, truncated at cap)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace abyss {

constexpr int kPad = 256;          // array padding (elements)
constexpr uint32_t kSpinLimit = 1u << 22;  // bounded mbarrier waits (~seconds at most)

// error bits written to the device status word
enum : int {
  kErrNone = 0,
  kErrTimeout = 1,      // an mbarrier wait ran out
  kErrOverflow = 2,     // some target's list exceeded cap (counts stay exact)
};

struct JSet {
  const double *px, *py, *pz;     // predicted positions
  const float4 *vm;               // (vx, vy, vz, m) FP32
  const double *pvx, *pvy, *pvz;  // predicted velocities FP64
  const double *mass;             // FP64 masses
  const double *r2nb;             // squared neighbour radii
  int n;
};

// One (target slice, j-range) unit of a batched launch over many clusters.
struct WorkItem {
  int t_begin;  // first entry in the order arrays
  int t_count;  // targets in the slice (<= threads x targets per thread)
  int j0, j1;   // j-range (the cluster's particles, or a chunk of them)
  int ch;       // chunk index of this j-range within the cluster
  int pad[3];
};

struct Work {
  const int *order_t;   // [m] target particle index, processing order
  const int *order_o;   // [m] output row, processing order
  int m;
  int n_chunks;         // S
  int chunk_len;        // j per chunk (multiple of the tile length)
  int cap;              // list capacity per (chunk, row) and per output row
  float eps2f;
  double eps2;
  int *lcnt;            // [m] neighbours found per target (atomic, exact)
  int *lst;             // [m][cap] neighbours in the order found
  double *part;         // [m][s_stride][6]
  int *status;          // error bits
  int *item_counter;    // work-queue head of the tile kernel
  int s_stride;         // partial-sum slots per row: part[(row * s_stride + ch) * 6]
  // batched launches (null/zero for a single cluster):
  const WorkItem *items;     // explicit work list
  const int *n_items_dev;    // its length, read on the device
  const int *m_dev;          // number of rows, read on the device
  const int *row_nchunks;    // chunks per row (else n_chunks)
  const int *row_joff;       // first particle of the row's cluster (lists are cluster-local)
  const int *row_jlen;       // particles of the row's cluster (else js.n)
  // anchor mode of a single cluster: per i-block anchor (x, y, z); null = the
  // block's first target
  const double *anchor = nullptr;
};

struct Outputs {
  const int *targets;   // [m] row -> target particle
  double *acc_reg, *jerk_reg, *acc_irr, *jerk_irr;  // [m][3]
  int *nnb;             // [m]
  int *list;            // [m][cap]
  int *overflow_rows;   // number of rows whose list exceeded cap
  int *ovf_list;        // [m] those rows, for the re-list pass
};

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// 1-D bulk copy global -> shared through the TMA engine (no multicast).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait on an mbarrier phase; returns false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < kSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// FP64 squared distance in the reference's operation order
// (ComputeAcceleration.cpp:253-261): r2 = 0 + dx*dx + dy*dy + dz*dz, no fused ops.
__device__ __forceinline__ double exact_r2(double xi, double yi, double zi, double xj, double yj,
                                           double zj) {
  const double dx = __dsub_rn(xj, xi), dy = __dsub_rn(yj, yi), dz = __dsub_rn(zj, zi);
  double r2 = __dmul_rn(dx, dx);
  r2 = __dadd_rn(r2, __dmul_rn(dy, dy));
  r2 = __dadd_rn(r2, __dmul_rn(dz, dz));
  return r2;
}

}  // namespace abyss
