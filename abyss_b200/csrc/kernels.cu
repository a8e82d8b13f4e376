// sm_100a kernels of the Ahmad-Cohen regular-force path.
//
//   predict_jset      device-side j prediction (UpdateParticle.cpp:37-59), FP64
//   target_bbox/curve_key/block_anchor  spatial ordering of targets and the
//                       i-block anchors of the anchor mode
//   reg_force_tile    i in registers, j-tiles through shared memory by TMA bulk
//                     copies, FP32 pair arithmetic with Kahan-folded tile sums,
//                     guarded FP32 neighbour test re-decided in FP64
//   reg_force_jmajor  lanes over j for very small active sets, two j per lane
//                     in FP32x2; guarded FP32 neighbour test re-decided in FP64
//   finalize_rows     FP64 cross-chunk sum, ordered list concatenation,
//                     FP64 irregular part over the final list
//
// Semantics follow the reference's CPU regular force
// (src_mpi/Particle/ComputeAcceleration.cpp:235-299): j ranges over all
// particles except the target; r2 < R_nb^2 (FP64, unsoftened) makes j a
// neighbour (irregular part, list in ascending j); every other j adds
// m r^-3 dx to the regular acceleration and m r^-3 (dv - 3 (dx.dv) dx / r^2)
// to the regular jerk, with r^2 softened by eps^2 in the force terms.
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cub/cub.cuh>

#include "abyss_internal.cuh"
#include "kernels.cuh"
#include "curve.cuh"

namespace abyss {

// ============================================================ prediction
// One thread per particle.  Intrinsics keep the reference's operation order
// with no fused multiply-add, so predicted values equal the host predictor's.
__global__ void predict_jset(int n, const double *__restrict__ x, const double *__restrict__ v,
                             const double *__restrict__ a0, const double *__restrict__ a1,
                             const double *__restrict__ t0, const double *__restrict__ mass,
                             double new_time, double time_scale, double *__restrict__ px,
                             double *__restrict__ py, double *__restrict__ pz,
                             double *__restrict__ pvx, double *__restrict__ pvy,
                             double *__restrict__ pvz, float4 *__restrict__ vm) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const double dt = __dmul_rn(__dsub_rn(new_time, t0[j]), time_scale);
    double p[3], q[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double xd = x[3 * j + d], vd = v[3 * j + d];
      if (dt == 0.0) {
        p[d] = xd;
        q[d] = vd;
      } else {
        const double a0d = a0[3 * j + d], a1d = a1[3 * j + d];
        double t = __dmul_rn(a1d, dt);
        t = __ddiv_rn(t, 3.0);
        t = __dadd_rn(t, a0d);
        t = __dmul_rn(t, dt);
        t = __ddiv_rn(t, 2.0);
        t = __dadd_rn(t, vd);
        t = __dmul_rn(t, dt);
        p[d] = __dadd_rn(t, xd);
        double u = __dmul_rn(a1d, dt);
        u = __ddiv_rn(u, 2.0);
        u = __dadd_rn(u, a0d);
        u = __dmul_rn(u, dt);
        q[d] = __dadd_rn(u, vd);
      }
    }
    px[j] = p[0];
    py[j] = p[1];
    pz[j] = p[2];
    pvx[j] = q[0];
    pvy[j] = q[1];
    pvz[j] = q[2];
    vm[j] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)mass[j]);
  }
}

// Prediction for a batched ensemble: particle j belongs to cluster cid[j]; only
// clusters flagged active this wave are predicted, each to its own time.
__global__ void predict_multi(int n, const int *__restrict__ cid, const int *__restrict__ active,
                              const double *__restrict__ new_time, const double *__restrict__ time_scale,
                              const double *__restrict__ x, const double *__restrict__ v,
                              const double *__restrict__ a0, const double *__restrict__ a1,
                              const double *__restrict__ t0, const double *__restrict__ mass,
                              double *__restrict__ px, double *__restrict__ py, double *__restrict__ pz,
                              double *__restrict__ pvx, double *__restrict__ pvy,
                              double *__restrict__ pvz, float4 *__restrict__ vm) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int k = cid[j];
    if (k < 0 || !active[k]) continue;  // padding between clusters, or an idle cluster
    const double dt = __dmul_rn(__dsub_rn(new_time[k], t0[j]), time_scale[k]);
    double p[3], q[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double xd = x[3 * j + d], vd = v[3 * j + d];
      if (dt == 0.0) {
        p[d] = xd;
        q[d] = vd;
      } else {
        const double a0d = a0[3 * j + d], a1d = a1[3 * j + d];
        double t = __dmul_rn(a1d, dt);
        t = __ddiv_rn(t, 3.0);
        t = __dadd_rn(t, a0d);
        t = __dmul_rn(t, dt);
        t = __ddiv_rn(t, 2.0);
        t = __dadd_rn(t, vd);
        t = __dmul_rn(t, dt);
        p[d] = __dadd_rn(t, xd);
        double u = __dmul_rn(a1d, dt);
        u = __ddiv_rn(u, 2.0);
        u = __dadd_rn(u, a0d);
        u = __dmul_rn(u, dt);
        q[d] = __dadd_rn(u, vd);
      }
    }
    px[j] = p[0];
    py[j] = p[1];
    pz[j] = p[2];
    pvx[j] = q[0];
    pvy[j] = q[1];
    pvz[j] = q[2];
    vm[j] = make_float4((float)q[0], (float)q[1], (float)q[2], (float)mass[j]);
  }
}

// j-set already predicted by the caller (reference-compatible SendToDevice):
// fill the FP32 (v, m) records from the FP64 arrays.
__global__ void pack_vm(int n, const double *__restrict__ pvx, const double *__restrict__ pvy,
                        const double *__restrict__ pvz, const double *__restrict__ mass,
                        float4 *__restrict__ vm) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    vm[j] = make_float4((float)pvx[j], (float)pvy[j], (float)pvz[j], (float)mass[j]);
}

// j-set given as predicted AoS [n][3] positions and velocities: split into the
// SoA FP64 arrays and the FP32 (v, m) records.
__global__ void unpack_predicted(int n, const double *__restrict__ pos, const double *__restrict__ vel,
                                 const double *__restrict__ mass, double *__restrict__ px,
                                 double *__restrict__ py, double *__restrict__ pz,
                                 double *__restrict__ pvx, double *__restrict__ pvy,
                                 double *__restrict__ pvz, float4 *__restrict__ vm) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    px[j] = pos[3 * j];
    py[j] = pos[3 * j + 1];
    pz[j] = pos[3 * j + 2];
    pvx[j] = vel[3 * j];
    pvy[j] = vel[3 * j + 1];
    pvz[j] = vel[3 * j + 2];
    vm[j] = make_float4((float)vel[3 * j], (float)vel[3 * j + 1], (float)vel[3 * j + 2], (float)mass[j]);
  }
}

// ============================================================ target ordering
__device__ __forceinline__ int ordered_int(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float from_ordered(int i) {
  return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff);
}

__global__ void target_bbox(int m, const int *__restrict__ targets, const double *__restrict__ px,
                            const double *__restrict__ py, const double *__restrict__ pz,
                            int *__restrict__ bbox /* [6]: min xyz, max xyz */) {
  int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < m; s += gridDim.x * blockDim.x) {
    const int t = targets[s];
    const int c[3] = {ordered_int((float)px[t]), ordered_int((float)py[t]), ordered_int((float)pz[t])};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      mn[d] = min(mn[d], c[d]);
      mx[d] = max(mx[d], c[d]);
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o > 0; o >>= 1) {
      mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
      mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      atomicMin(&bbox[d], mn[d]);
      atomicMax(&bbox[3 + d], mx[d]);
    }
  }
}

// Hilbert key of each target on a 1024^3 grid over the targets' FP32 bounding box.
__global__ void target_curve_key(int m, const int *__restrict__ targets, const double *__restrict__ px,
                                 const double *__restrict__ py, const double *__restrict__ pz,
                                 const int *__restrict__ bbox, uint32_t *__restrict__ keys,
                                 int *__restrict__ rows) {
  const float lo[3] = {from_ordered(bbox[0]), from_ordered(bbox[1]), from_ordered(bbox[2])};
  const float hi[3] = {from_ordered(bbox[3]), from_ordered(bbox[4]), from_ordered(bbox[5])};
  float sc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) sc[d] = hi[d] > lo[d] ? 1023.0f / (hi[d] - lo[d]) : 0.0f;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < m; s += gridDim.x * blockDim.x) {
    const int t = targets[s];
    const float c[3] = {(float)px[t], (float)py[t], (float)pz[t]};
    uint32_t q[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float f = (c[d] - lo[d]) * sc[d];
      f = fminf(fmaxf(f, 0.0f), 1023.0f);
      q[d] = (uint32_t)f;
    }
    keys[s] = hilbert_key10(q[0], q[1], q[2]);
    rows[s] = s;
  }
}

// Anchor of each i-block of `per_block` consecutive slots of the processing
// order: the centre of the block's FP64 bounding box, so that no target of the
// block is further from it than half the block's extent per axis.  One warp
// per block; min/max are exact, so the anchor does not depend on the order of
// the reduction.
__global__ void block_anchor(int m, int per_block, const int *__restrict__ order_t,
                             const double *__restrict__ px, const double *__restrict__ py,
                             const double *__restrict__ pz, double *__restrict__ anchor) {
  const int lane = threadIdx.x & 31;
  const int nblk = (m + per_block - 1) / per_block;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nblk; b += (gridDim.x * blockDim.x) >> 5) {
    const int s0 = b * per_block, s1 = min(m, s0 + per_block);
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int s = s0 + lane; s < s1; s += 32) {
      const int t = order_t[s];
      const double c[3] = {px[t], py[t], pz[t]};
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        lo[d] = fmin(lo[d], c[d]);
        hi[d] = fmax(hi[d], c[d]);
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d)
      for (int o = 16; o > 0; o >>= 1) {
        lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
        hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
      }
    if (lane < 3) {
      const double l = lane == 0 ? lo[0] : lane == 1 ? lo[1] : lo[2];
      const double h = lane == 0 ? hi[0] : lane == 1 ? hi[1] : hi[2];
      anchor[3 * (size_t)b + lane] = __dadd_rn(l, __dmul_rn(0.5, __dsub_rn(h, l)));
    }
  }
}

__global__ void gather_order(int m, const int *__restrict__ targets, const int *__restrict__ rows_sorted,
                             int *__restrict__ order_t, int *__restrict__ order_o) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < m; s += gridDim.x * blockDim.x) {
    const int r = rows_sorted[s];
    order_o[s] = r;
    order_t[s] = targets[r];
  }
}

__global__ void iota_kernel(int m, int *__restrict__ out) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < m; s += gridDim.x * blockDim.x) out[s] = s;
}

// ============================================================ pair arithmetic
// Shared by the fast path and the slow (candidate) path so that both see the
// very same FP32 r^2: explicit round-to-nearest intrinsics forbid the compiler
// from contracting or reordering either copy.
struct PairGeom {
  float dx, dy, dz, dvx, dvy, dvz, r2, rv;
};

__device__ __forceinline__ PairGeom pair_geom(float xj, float yj, float zj, float vxj, float vyj,
                                              float vzj, float xi, float yi, float zi, float vxi,
                                              float vyi, float vzi, float eps2) {
  PairGeom g;
  g.dx = __fsub_rn(xj, xi);
  g.dy = __fsub_rn(yj, yi);
  g.dz = __fsub_rn(zj, zi);
  g.dvx = __fsub_rn(vxj, vxi);
  g.dvy = __fsub_rn(vyj, vyi);
  g.dvz = __fsub_rn(vzj, vzi);
  g.r2 = __fmaf_rn(g.dx, g.dx, __fmaf_rn(g.dy, g.dy, __fmaf_rn(g.dz, g.dz, eps2)));
  g.rv = __fmaf_rn(g.dx, g.dvx, __fmaf_rn(g.dy, g.dvy, __fmul_rn(g.dz, g.dvz)));
  return g;
}

// Double-single differencing: d = (hj - hi) + (lj - li).
__device__ __forceinline__ PairGeom pair_geom_ds(float xj, float yj, float zj, float xjl, float yjl,
                                                 float zjl, float vxj, float vyj, float vzj,
                                                 float xi, float yi, float zi, float xil, float yil,
                                                 float zil, float vxi, float vyi, float vzi,
                                                 float eps2) {
  PairGeom g;
  g.dx = __fadd_rn(__fsub_rn(xj, xi), __fsub_rn(xjl, xil));
  g.dy = __fadd_rn(__fsub_rn(yj, yi), __fsub_rn(yjl, yil));
  g.dz = __fadd_rn(__fsub_rn(zj, zi), __fsub_rn(zjl, zil));
  g.dvx = __fsub_rn(vxj, vxi);
  g.dvy = __fsub_rn(vyj, vyi);
  g.dvz = __fsub_rn(vzj, vzi);
  g.r2 = __fmaf_rn(g.dx, g.dx, __fmaf_rn(g.dy, g.dy, __fmaf_rn(g.dz, g.dz, eps2)));
  g.rv = __fmaf_rn(g.dx, g.dvx, __fmaf_rn(g.dy, g.dvy, __fmul_rn(g.dz, g.dvz)));
  return g;
}

// acc += m r^-3 d;  jerk += m r^-3 (dv - 3 (d.dv)/r^2 d)  with rinv possibly masked to 0.
__device__ __forceinline__ void pair_accum(const PairGeom &g, float mj, float rinv, float *p) {
  const float q = rinv * rinv;
  const float mr3 = mj * rinv * q;
  const float al = -3.0f * g.rv * q;
  p[0] = fmaf(mr3, g.dx, p[0]);
  p[1] = fmaf(mr3, g.dy, p[1]);
  p[2] = fmaf(mr3, g.dz, p[2]);
  p[3] = fmaf(mr3, fmaf(al, g.dx, g.dvx), p[3]);
  p[4] = fmaf(mr3, fmaf(al, g.dy, g.dvy), p[4]);
  p[5] = fmaf(mr3, fmaf(al, g.dz, g.dvz), p[5]);
}

// ============================================================ tile kernel
template <int TJ>
struct __align__(16) JStage {
  double x[TJ];
  double y[TJ];
  double z[TJ];
  float4 vm[TJ];
};

template <int TJ>
__device__ __forceinline__ void issue_tile(JStage<TJ> *st, uint64_t *bar, const JSet &js, int jt0,
                                           int j1) {
  // The even part of the tile moves by TMA bulk copies (16-byte aligned FP64
  // sources: callers keep jt0 even, and the host checks every j-range); an odd
  // last element is loaded by this thread before the arrive, whose release
  // ordering makes it visible to the waiting threads.  Nothing past j1 is read.
  const int cnt = min(TJ, j1 - jt0);
  const int ce = cnt & ~1;
  if (cnt & 1) {
    st->x[ce] = js.px[jt0 + ce];
    st->y[ce] = js.py[jt0 + ce];
    st->z[ce] = js.pz[jt0 + ce];
    st->vm[ce] = js.vm[jt0 + ce];
  }
  const uint32_t b8 = (uint32_t)ce * 8u, b16 = (uint32_t)ce * 16u;
  mbar_arrive_expect_tx(bar, 3u * b8 + b16);
  if (ce > 0) {
    bulk_g2s(st->x, js.px + jt0, b8, bar);
    bulk_g2s(st->y, js.py + jt0, b8, bar);
    bulk_g2s(st->z, js.pz + jt0, b8, bar);
    bulk_g2s(st->vm, js.vm + jt0, b16, bar);
  }
}

// Packed (FP32x2) pair arithmetic: sm_100's __fadd2_rn / __fmul2_rn / __ffma2_rn
// carry the pair arithmetic of two targets in one instruction; only rsqrt and
// the candidate select stay scalar.  Target coordinates are held negated so
// that every difference is an addition.
struct PairGeom2 {
  float2 dx, dy, dz, dvx, dvy, dvz, r2, rv;
};

__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }

__device__ __forceinline__ PairGeom2 pair_geom2(float2 xj, float2 yj, float2 zj, float2 vxj, float2 vyj,
                                                float2 vzj, float2 nxi, float2 nyi, float2 nzi,
                                                float2 nvxi, float2 nvyi, float2 nvzi, float2 eps2) {
  PairGeom2 g;
  g.dx = __fadd2_rn(xj, nxi);
  g.dy = __fadd2_rn(yj, nyi);
  g.dz = __fadd2_rn(zj, nzi);
  g.dvx = __fadd2_rn(vxj, nvxi);
  g.dvy = __fadd2_rn(vyj, nvyi);
  g.dvz = __fadd2_rn(vzj, nvzi);
  g.r2 = __ffma2_rn(g.dx, g.dx, __ffma2_rn(g.dy, g.dy, __ffma2_rn(g.dz, g.dz, eps2)));
  g.rv = __ffma2_rn(g.dx, g.dvx, __ffma2_rn(g.dy, g.dvy, __fmul2_rn(g.dz, g.dvz)));
  return g;
}

// double-single differencing: d = (hj - hi) + (lj - li), with hi, li held negated
__device__ __forceinline__ PairGeom2 pair_geom2_ds(float2 xj, float2 yj, float2 zj, float2 xjl, float2 yjl,
                                                   float2 zjl, float2 vxj, float2 vyj, float2 vzj,
                                                   float2 nxi, float2 nyi, float2 nzi, float2 nxil,
                                                   float2 nyil, float2 nzil, float2 nvxi, float2 nvyi,
                                                   float2 nvzi, float2 eps2) {
  PairGeom2 g;
  g.dx = __fadd2_rn(__fadd2_rn(xj, nxi), __fadd2_rn(xjl, nxil));
  g.dy = __fadd2_rn(__fadd2_rn(yj, nyi), __fadd2_rn(yjl, nyil));
  g.dz = __fadd2_rn(__fadd2_rn(zj, nzi), __fadd2_rn(zjl, nzil));
  g.dvx = __fadd2_rn(vxj, nvxi);
  g.dvy = __fadd2_rn(vyj, nvyi);
  g.dvz = __fadd2_rn(vzj, nvzi);
  g.r2 = __ffma2_rn(g.dx, g.dx, __ffma2_rn(g.dy, g.dy, __ffma2_rn(g.dz, g.dz, eps2)));
  g.rv = __ffma2_rn(g.dx, g.dvx, __ffma2_rn(g.dy, g.dvy, __fmul2_rn(g.dz, g.dvz)));
  return g;
}

__device__ __forceinline__ void pair_accum2(const PairGeom2 &g, float2 mj, float2 rinv, float2 *p) {
  const float2 q = __fmul2_rn(rinv, rinv);
  const float2 mr3 = __fmul2_rn(__fmul2_rn(mj, rinv), q);
  const float2 al = __fmul2_rn(__fmul2_rn(dup2(-3.0f), g.rv), q);
  p[0] = __ffma2_rn(mr3, g.dx, p[0]);
  p[1] = __ffma2_rn(mr3, g.dy, p[1]);
  p[2] = __ffma2_rn(mr3, g.dz, p[2]);
  p[3] = __ffma2_rn(mr3, __ffma2_rn(al, g.dx, g.dvx), p[3]);
  p[4] = __ffma2_rn(mr3, __ffma2_rn(al, g.dy, g.dvy), p[4]);
  p[5] = __ffma2_rn(mr3, __ffma2_rn(al, g.dz, g.dvz), p[5]);
}

// A j-particle as packed operands: each value of the compute buffer's float4
// records broadcast to both halves of a float2.
struct JPair2 {
  float2 x, y, z, m, vx, vy, vz, lx, ly, lz;
};

template <bool ANCHOR>
__device__ __forceinline__ JPair2 jpair2_of(const float4 &P, const float4 &V, const float4 &L) {
  JPair2 J;
  J.x = dup2(P.x);
  J.y = dup2(P.y);
  J.z = dup2(P.z);
  J.m = dup2(P.w);
  J.vx = dup2(V.x);
  J.vy = dup2(V.y);
  J.vz = dup2(V.z);
  if (!ANCHOR) {
    J.lx = dup2(L.x);
    J.ly = dup2(L.y);
    J.lz = dup2(L.z);
  } else {
    J.lx = J.ly = J.lz = make_float2(0.f, 0.f);
  }
  return J;
}

// Geometry of j against the target pair q (targets 2q, 2q+1) held negated.
template <bool ANCHOR, int IPT>
__device__ __forceinline__ PairGeom2 geom2_of(const JPair2 &J, int q, const float (&hx)[IPT],
                                              const float (&hy)[IPT], const float (&hz)[IPT],
                                              const float (&lx)[IPT], const float (&ly)[IPT],
                                              const float (&lz)[IPT], const float (&vx)[IPT],
                                              const float (&vy)[IPT], const float (&vz)[IPT], float2 eps2) {
  const int k0 = 2 * q, k1 = 2 * q + 1;
  if (ANCHOR)
    return pair_geom2(J.x, J.y, J.z, J.vx, J.vy, J.vz, make_float2(hx[k0], hx[k1]), make_float2(hy[k0], hy[k1]),
                      make_float2(hz[k0], hz[k1]), make_float2(vx[k0], vx[k1]), make_float2(vy[k0], vy[k1]),
                      make_float2(vz[k0], vz[k1]), eps2);
  return pair_geom2_ds(J.x, J.y, J.z, J.lx, J.ly, J.lz, J.vx, J.vy, J.vz, make_float2(hx[k0], hx[k1]),
                       make_float2(hy[k0], hy[k1]), make_float2(hz[k0], hz[k1]), make_float2(lx[k0], lx[k1]),
                       make_float2(ly[k0], ly[k1]), make_float2(lz[k0], lz[k1]), make_float2(vx[k0], vx[k1]),
                       make_float2(vy[k0], vy[k1]), make_float2(vz[k0], vz[k1]), eps2);
}

// Shared-memory layout of the tile kernel (dynamic).
template <int NT, int IPT, int TJ, int NST, bool ANCHOR, bool PACK>
struct TileLayout {
  static constexpr int TJP = TJ + 4;           // compute buffer incl. pad entries
  // float4 records per j: (x,y,z,m) (vx,vy,vz,-) [+ (xl,yl,zl,-) with double-single].
  static constexpr int CW = ANCHOR ? 2 : 3;
  static constexpr size_t stage = 0;
  static constexpr size_t cbuf = stage + NST * sizeof(JStage<TJ>);
  static constexpr size_t kahan = cbuf + 2 * CW * TJP * sizeof(float4);  // float [IPT*12][NT]
  static constexpr size_t tgt = kahan + (size_t)IPT * 12 * NT * sizeof(float);  // int [IPT][NT]
  static constexpr size_t rows = tgt + (size_t)IPT * NT * sizeof(int);         // int [IPT][NT]
  static constexpr size_t bar = (rows + (size_t)IPT * NT * sizeof(int) + 7) / 8 * 8;
  static constexpr size_t item = bar + NST * sizeof(uint64_t);
  static constexpr size_t bytes = item + 16;
};

// Regular force over a work queue of (i-block, j-chunk) items.  Each CTA takes
// items from a device counter (grid = SMs x resident CTAs); an item streams its
// j-chunk through NST shared-memory stages filled by TMA bulk copies, converts
// each tile to FP32 offsets (anchor-relative or double-single) once per CTA and
// runs the pair loop with IPT targets per thread in registers.  Pairs inside a
// guard band of R_nb are masked in the fast path and re-decided with the FP64
// test in a warp-uniform slow path (list entry, or regular contribution).
// Tile partials are FP32; they are folded into Kahan-compensated FP32 sums kept
// in shared memory, and written per (chunk, target) for the FP64 finalize.
//
// JW > 1 (warps sharing targets): the block's JW warps hold the same 32 x IPT
// targets and each takes every JW-th group of 32 j of a tile, so that a small
// active set still fills the SMs with warps; at the end of an item warp 0 adds
// the warps' sums in FP64 in warp order.
//
// PJ (one target per thread): two j per step as the two halves of the FP32x2
// operands, so that the pair arithmetic of a single target also runs packed;
// the halves' tile partials are added at the end of the tile.
template <int NT, int IPT, int TJ, int NST, bool ANCHOR, bool PACK, int UNR, int MINB, int JW = 1, bool PJ = false>
__global__ void __launch_bounds__(NT, MINB) reg_force_tile(JSet js, Work w, int n_iblocks) {
  static_assert(JW == 1 || NT == 32 * JW, "warps sharing targets: one target slot per lane");
  static_assert(!PJ || (IPT == 1 && !PACK), "two j per step: one target per thread, scalar otherwise");
  using LY = TileLayout<NT, IPT, TJ, NST, ANCHOR, PACK>;
  constexpr int TS = JW > 1 ? 32 : NT;  // target slots per k (per lane, or per thread)
  constexpr int TJP = LY::TJP;
  constexpr int CW = LY::CW;
  // With PACK, targets 0 .. NPK-1 run in pairs on FP32x2 instructions and an odd
  // last target on scalar ones; without, every target is scalar.
  constexpr int NPK = PACK ? 2 * (IPT / 2) : 0;
  constexpr int PP = NPK > 0 ? NPK / 2 : 1;
  static_assert(32 % UNR == 0 && UNR <= 4, "a 32-j group is whole unroll steps; pad covers UNR - 1");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  JStage<TJ> *st = reinterpret_cast<JStage<TJ> *>(smem_raw + LY::stage);
  float4 *cbuf = reinterpret_cast<float4 *>(smem_raw + LY::cbuf);
  float *ksm = reinterpret_cast<float *>(smem_raw + LY::kahan);
  int *s_ti = reinterpret_cast<int *>(smem_raw + LY::tgt);
  int *s_row = reinterpret_cast<int *>(smem_raw + LY::rows);
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + LY::bar);
  int *s_item = reinterpret_cast<int *>(smem_raw + LY::item);
  const int tid = threadIdx.x;
  const int sl = JW > 1 ? (tid & 31) : tid;  // this thread's target slot
  const int wid = tid >> 5;
  const unsigned FULL = 0xffffffffu;

  if (tid == 0) {
    for (int s = 0; s < NST; ++s) mbar_init(&bar[s], 1);
    fence_barrier_init();
  }
  __syncthreads();

  uint32_t g_cons = 0, g_issue = 0;
  const int n_items = w.items ? *w.n_items_dev : n_iblocks * w.n_chunks;
  const int m_rows = w.m_dev ? *w.m_dev : w.m;
  for (;;) {
    if (tid == 0) *s_item = atomicAdd(w.item_counter, 1);
    __syncthreads();
    const int item = *s_item;
    if (item >= n_items) break;
    int base, count, ch, j0, j1;
    if (w.items) {
      const WorkItem it = w.items[item];
      base = it.t_begin;
      count = it.t_count;
      ch = it.ch;
      j0 = it.j0;
      j1 = it.j1;
    } else {
      const int ib = item / w.n_chunks;
      ch = item - ib * w.n_chunks;
      base = ib * TS * IPT;
      count = min(TS * IPT, m_rows - base);
      j0 = ch * w.chunk_len;
      j1 = min(js.n, j0 + w.chunk_len);
    }
    const int ntile = (j1 - j0 + TJ - 1) / TJ;

    if (tid == 0) {
      const int pro = min(NST, ntile);
      for (int p = 0; p < pro; ++p, ++g_issue)
        issue_tile<TJ>(&st[g_issue % NST], &bar[g_issue % NST], js, j0 + p * TJ, j1);
    }

    // ---- targets of this block into registers (coordinates) and shared memory (indices)
    double ax = 0.0, ay = 0.0, az = 0.0;
    if (ANCHOR) {
      if (w.anchor && !w.items) {  // the i-block's bounding-box centre
        const double *a = w.anchor + 3 * (size_t)(base / (TS * IPT));
        ax = a[0];
        ay = a[1];
        az = a[2];
      } else {  // the block's first target
        const int t0 = w.order_t[base];
        ax = js.px[t0];
        ay = js.py[t0];
        az = js.pz[t0];
      }
    }
    // scalar layout: [k]; packed layout: [k/2].{x,y}; coordinates held negated
    float hx[IPT], hy[IPT], hz[IPT], lx[IPT], ly[IPT], lz[IPT], vx[IPT], vy[IPT], vz[IPT], r2g[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      const int s = base + k * TS + sl;
      const bool valid = k * TS + sl < count;
      const int si = valid ? s : base;
      const int t = w.order_t[si];
      if (JW == 1 || wid == 0) {
        s_ti[k * TS + sl] = t;
        s_row[k * TS + sl] = valid ? w.order_o[si] : -1;
      }
      const double X = js.px[t], Y = js.py[t], Z = js.pz[t];
      double spread = 0.0;
      if (ANCHOR) {
        hx[k] = -(float)(X - ax);
        hy[k] = -(float)(Y - ay);
        hz[k] = -(float)(Z - az);
        lx[k] = ly[k] = lz[k] = 0.0f;
        spread = fmax(fabs(X - ax), fmax(fabs(Y - ay), fabs(Z - az)));
      } else {
        const float fx = (float)X, fy = (float)Y, fz = (float)Z;
        hx[k] = -fx;
        hy[k] = -fy;
        hz[k] = -fz;
        lx[k] = -(float)(X - (double)fx);
        ly[k] = -(float)(Y - (double)fy);
        lz[k] = -(float)(Z - (double)fz);
      }
      const float4 vmi = js.vm[t];
      vx[k] = -vmi.x;
      vy[k] = -vmi.y;
      vz[k] = -vmi.z;
      // Candidate threshold: every FP64 neighbour (r2 < R2) passes the FP32
      // test r2f < r2g.  FP32 offsets err by at most ~2^-23 (|d| + 2 spread)
      // per component; the margin below covers that many times over.
      const double R2 = js.r2nb[t];
      const double R = sqrt(fmax(R2, 0.0));
      const double Rg = R * (1.0 + 0x1p-17) + 0x1p-19 * spread + 1e-30;
      float g = __double2float_ru(Rg * Rg + w.eps2);
      g = fmaxf(g, nextafterf(w.eps2f, FLT_MAX));  // the self pair (r2 = eps2) is always a candidate
      r2g[k] = valid ? g : -1.0f;
#pragma unroll
      for (int c = 0; c < 12; ++c) ksm[(k * 12 + c) * NT + tid] = 0.0f;
    }
    const float2 eps2v = dup2(w.eps2f);

    // ---- stream the chunk's j-tiles
    for (int t = 0; t < ntile; ++t, ++g_cons) {
      const int stg = g_cons % NST;
      const bool ok = mbar_wait(&bar[stg], (g_cons / NST) & 1u);
      const int jt0 = j0 + t * TJ;
      const int cnt = min(TJ, j1 - jt0);
      float4 *cb = cbuf + (g_cons & 1u) * CW * TJP;
      for (int jj = tid; jj < TJP; jj += NT) {
        const bool real = jj < cnt && ok;
        double X = 0.0, Y = 0.0, Z = 0.0;
        float4 vmj = make_float4(0.f, 0.f, 0.f, 0.f);
        if (real) {
          X = st[stg].x[jj];
          Y = st[stg].y[jj];
          Z = st[stg].z[jj];
          vmj = st[stg].vm[jj];
        }
        // pad entries are massless and far away: never a candidate, contribute 0
        float fx, fy, fz, lxj = 0.0f, lyj = 0.0f, lzj = 0.0f;
        if (!real) {
          fx = fy = fz = 1e30f;
        } else if (ANCHOR) {
          fx = (float)(X - ax);
          fy = (float)(Y - ay);
          fz = (float)(Z - az);
        } else {
          fx = (float)X;
          fy = (float)Y;
          fz = (float)Z;
          lxj = (float)(X - (double)fx);
          lyj = (float)(Y - (double)fy);
          lzj = (float)(Z - (double)fz);
        }
        cb[jj] = make_float4(fx, fy, fz, vmj.w);
        cb[TJP + jj] = make_float4(vmj.x, vmj.y, vmj.z, 0.0f);
        if (!ANCHOR) cb[2 * TJP + jj] = make_float4(lxj, lyj, lzj, 0.0f);
      }
      if (!__syncthreads_and(ok)) {
        if (tid == 0) {
          atomicOr(w.status, kErrTimeout);
          // let the copies already in flight land before the CTA leaves
          for (uint32_t g = g_cons; g < g_issue; ++g) (void)mbar_wait(&bar[g % NST], (g / NST) & 1u);
        }
        __syncthreads();
        return;
      }
      if (tid == 0 && t + NST < ntile) {
        issue_tile<TJ>(&st[g_issue % NST], &bar[g_issue % NST], js, j0 + (t + NST) * TJ, j1);
        ++g_issue;
      }

      float p[IPT][6];  // scalar tile partials
      float2 p2[PP][6]; // packed tile partials
      float2 pj[6];     // PJ: the two j streams of target 0
#pragma unroll
      for (int k = 0; k < IPT; ++k)
#pragma unroll
        for (int c = 0; c < 6; ++c) p[k][c] = 0.0f;
#pragma unroll
      for (int q = 0; q < PP; ++q)
#pragma unroll
        for (int c = 0; c < 6; ++c) p2[q][c] = make_float2(0.0f, 0.0f);
#pragma unroll
      for (int c = 0; c < 6; ++c) pj[c] = make_float2(0.0f, 0.0f);

      // Fast path, 32 j at a time: every pair is accumulated with candidates
      // (pairs inside the guard band of R_nb) masked to 0, and each thread sets
      // bit l of cbits when j = g0 + l gave it a candidate.  No branch depends on
      // the data, so the j iterations schedule freely.  Up to UNR - 1 pad entries
      // past cnt may be visited: they are far away and massless, never
      // candidates, and contribute exactly 0.
      for (int g0 = JW > 1 ? 32 * wid : 0; g0 < cnt; g0 += 32 * JW) {
        const int gl = min(32, cnt - g0);
        unsigned cbits = 0u;
        if constexpr (PJ) {
          // j = g0 + l and g0 + l + 1 in the two halves (an odd last one pairs
          // with a pad entry)
          for (int l = 0; l < gl; l += 2) {
            const int jl = g0 + l;
            const float4 P0 = cb[jl], P1 = cb[jl + 1];
            const float4 V0 = cb[TJP + jl], V1 = cb[TJP + jl + 1];
            PairGeom2 g;
            if (ANCHOR) {
              g = pair_geom2(make_float2(P0.x, P1.x), make_float2(P0.y, P1.y), make_float2(P0.z, P1.z),
                             make_float2(V0.x, V1.x), make_float2(V0.y, V1.y), make_float2(V0.z, V1.z), dup2(hx[0]),
                             dup2(hy[0]), dup2(hz[0]), dup2(vx[0]), dup2(vy[0]), dup2(vz[0]), eps2v);
            } else {
              const float4 L0 = cb[2 * TJP + jl], L1 = cb[2 * TJP + jl + 1];
              g = pair_geom2_ds(make_float2(P0.x, P1.x), make_float2(P0.y, P1.y), make_float2(P0.z, P1.z),
                                make_float2(L0.x, L1.x), make_float2(L0.y, L1.y), make_float2(L0.z, L1.z),
                                make_float2(V0.x, V1.x), make_float2(V0.y, V1.y), make_float2(V0.z, V1.z), dup2(hx[0]),
                                dup2(hy[0]), dup2(hz[0]), dup2(lx[0]), dup2(ly[0]), dup2(lz[0]), dup2(vx[0]),
                                dup2(vy[0]), dup2(vz[0]), eps2v);
            }
            const bool c0 = g.r2.x < r2g[0];
            const bool c1 = g.r2.y < r2g[0];
            float2 ri;
            ri.x = c0 ? 0.0f : rsqrtf(g.r2.x);
            ri.y = c1 ? 0.0f : rsqrtf(g.r2.y);
            pair_accum2(g, make_float2(P0.w, P1.w), ri, pj);
            cbits |= ((unsigned)c0 << l) | ((unsigned)c1 << (l + 1));
          }
        } else
        for (int l = 0; l < gl; l += UNR) {
#pragma unroll
          for (int u = 0; u < UNR; ++u) {
            const int jl = g0 + l + u;
            bool any = false;
            const float4 P = cb[jl];
            const float4 V = cb[TJP + jl];
            const float4 L = ANCHOR ? make_float4(0.f, 0.f, 0.f, 0.f) : cb[2 * TJP + jl];
            if constexpr (NPK > 0) {
              const JPair2 J = jpair2_of<ANCHOR>(P, V, L);
#pragma unroll
              for (int q = 0; q < NPK / 2; ++q) {
                const PairGeom2 g = geom2_of<ANCHOR>(J, q, hx, hy, hz, lx, ly, lz, vx, vy, vz, eps2v);
                const bool c0 = g.r2.x < r2g[2 * q];
                const bool c1 = g.r2.y < r2g[2 * q + 1];
                float2 ri;
                ri.x = c0 ? 0.0f : rsqrtf(g.r2.x);
                ri.y = c1 ? 0.0f : rsqrtf(g.r2.y);
                any |= (c0 | c1);
                pair_accum2(g, J.m, ri, p2[q]);
              }
            }
#pragma unroll
            for (int k = NPK; k < IPT; ++k) {
              const PairGeom gg =
                  ANCHOR ? pair_geom(P.x, P.y, P.z, V.x, V.y, V.z, -hx[k], -hy[k], -hz[k], -vx[k], -vy[k],
                                     -vz[k], w.eps2f)
                         : pair_geom_ds(P.x, P.y, P.z, L.x, L.y, L.z, V.x, V.y, V.z, -hx[k], -hy[k], -hz[k],
                                        -lx[k], -ly[k], -lz[k], -vx[k], -vy[k], -vz[k], w.eps2f);
              const bool cand = gg.r2 < r2g[k];
              float rinv = rsqrtf(gg.r2);
              rinv = cand ? 0.0f : rinv;
              any |= cand;
              pair_accum(gg, P.w, rinv, p[k]);
            }
            cbits |= (unsigned)any << (l + u);
          }
        }
        // Slow path: every j of the group that gave any thread of the warp a
        // candidate is re-decided with the FP64 test (a warp-uniform loop over
        // the set bits, in ascending j).
        unsigned wbits = __reduce_or_sync(FULL, cbits);
        while (wbits) {
          const int jl = g0 + __ffs(wbits) - 1;
          wbits &= wbits - 1u;
          if (jl >= cnt) break;
          const int jg = jt0 + jl;
          const float4 P = cb[jl];
          const float4 V = cb[TJP + jl];
          const float4 L = ANCHOR ? make_float4(0.f, 0.f, 0.f, 0.f) : cb[2 * TJP + jl];
          const float mj = P.w;
#pragma unroll
          for (int k = 0; k < IPT; ++k) {
            float r2k;
            PairGeom2 g2;
            PairGeom gg;
            if (k < NPK) {
              g2 = geom2_of<ANCHOR>(jpair2_of<ANCHOR>(P, V, L), k >> 1, hx, hy, hz, lx, ly, lz, vx, vy, vz,
                                    eps2v);
              r2k = (k & 1) ? g2.r2.y : g2.r2.x;
            } else {
              gg = ANCHOR ? pair_geom(P.x, P.y, P.z, V.x, V.y, V.z, -hx[k], -hy[k], -hz[k], -vx[k], -vy[k],
                                      -vz[k], w.eps2f)
                          : pair_geom_ds(P.x, P.y, P.z, L.x, L.y, L.z, V.x, V.y, V.z, -hx[k], -hy[k], -hz[k],
                                         -lx[k], -ly[k], -lz[k], -vx[k], -vy[k], -vz[k], w.eps2f);
              r2k = gg.r2;
            }
            if (!(r2k < r2g[k])) continue;
            const int ti = s_ti[k * TS + sl];
            if (jg == ti) continue;
            const double r2e = exact_r2(js.px[ti], js.py[ti], js.pz[ti], js.px[jg], js.py[jg], js.pz[jg]);
            if (r2e < js.r2nb[ti]) {
              const int row = s_row[k * TS + sl];
              const int pos = atomicAdd(&w.lcnt[row], 1);
              if (pos < w.cap) w.lst[(size_t)row * w.cap + pos] = jg;
            } else {
              const float rr = rsqrtf(r2k);
              if (k < NPK)
                pair_accum2(g2, dup2(mj), (k & 1) ? make_float2(0.0f, rr) : make_float2(rr, 0.0f), p2[k >> 1]);
              else
                pair_accum(gg, mj, rr, p[k]);
            }
          }
        }
      }
      // Kahan fold of the tile partials into the shared-memory sums
#pragma unroll
      for (int k = 0; k < IPT; ++k)
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          float pv;
          if (k < NPK)
            pv = (k & 1) ? p2[k >> 1][c].y : p2[k >> 1][c].x;
          else if (PJ)
            pv = __fadd_rn(__fadd_rn(pj[c].x, pj[c].y), p[k][c]);
          else
            pv = p[k][c];
          float *sp = &ksm[(k * 12 + c) * NT + tid];
          float *cp = &ksm[(k * 12 + 6 + c) * NT + tid];
          const float ssum = *sp, comp = *cp;
          const float y = __fsub_rn(pv, comp);
          const float tt = __fadd_rn(ssum, y);
          *cp = __fsub_rn(__fsub_rn(tt, ssum), y);
          *sp = tt;
        }
    }

    if constexpr (JW == 1) {
#pragma unroll
      for (int k = 0; k < IPT; ++k) {
        const int row = s_row[k * NT + tid];
        if (row < 0) continue;
        double *dst = w.part + ((size_t)row * w.s_stride + ch) * 6;
#pragma unroll
        for (int c = 0; c < 6; ++c)
          dst[c] = (double)ksm[(k * 12 + c) * NT + tid] - (double)ksm[(k * 12 + 6 + c) * NT + tid];
      }
    } else {
      // the warps' compensated sums of each target, in FP64 in warp order
      __syncthreads();
      if (wid == 0) {
#pragma unroll
        for (int k = 0; k < IPT; ++k) {
          const int row = s_row[k * TS + sl];
          if (row < 0) continue;
          double *dst = w.part + ((size_t)row * w.s_stride + ch) * 6;
#pragma unroll
          for (int c = 0; c < 6; ++c) {
            double v = 0.0;
#pragma unroll
            for (int q = 0; q < JW; ++q)
              v += (double)ksm[(k * 12 + c) * NT + 32 * q + sl] - (double)ksm[(k * 12 + 6 + c) * NT + 32 * q + sl];
            dst[c] = v;
          }
        }
      }
      __syncthreads();  // the next item's set-up rewrites the sums and the target slots
    }
  }
}

// ============================================================ j-major kernel
// For very small active sets: lanes over j, every lane holding the same MI
// targets.  A block of kJmWarps warps covers one j-chunk (its partials are one
// column of the chunk-partial array); each warp takes a contiguous sub-chunk of
// Lw particles (a multiple of 64) and each lane two j per step, j and j + 32,
// as the halves of FP32x2 operands with double-single differencing.  Pairs
// inside the guard band of R_nb are masked in that fast path and re-decided by
// their own lane with the exact FP64 test: a neighbour is appended to the
// target's list (one atomic per neighbour), any other pair adds its unmasked
// FP32 contribution.  Lane halves and lanes are summed in FP64 in a fixed tree,
// warps in a fixed order, so a launch is deterministic.
constexpr int kJmWarps = 4;

template <int NT>
__device__ void finalize_row_block(const JSet &js, const Work &w, const Outputs &o, int sort_cap, int r,
                                   int *fin_smem, double (*red)[6], int *s_nl_total);

template <int MI>
__global__ void __launch_bounds__(32 * kJmWarps, MI <= 2 ? 5 : 1) reg_force_jmajor(JSet js, Work w, Outputs o, int Lw,
                                                                  int fuse_sort_cap) {
  __shared__ double s_red[kJmWarps][MI][6];
  const unsigned FULL = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ch = blockIdx.x;
  const int jw0 = min(js.n, (ch * kJmWarps + warp) * Lw);
  const int jw1 = min(js.n, jw0 + Lw);
  const float2 eps2v = dup2(w.eps2f);
  for (int ig = 0; ig < w.m; ig += MI) {
    // j records, two per lane a step; a pad is massless and far away: never a
    // candidate, adds 0.  The next step's records are loaded before this
    // step's arithmetic, so that a warp keeps two steps of loads in flight;
    // the first step's are issued before the targets' loads, which they do not
    // depend on.
    double nX0 = 1e30, nY0 = 1e30, nZ0 = 1e30, nX1 = 1e30, nY1 = 1e30, nZ1 = 1e30;
    float4 nV0 = make_float4(0.f, 0.f, 0.f, 0.f), nV1 = nV0;
    if (jw0 + lane < jw1) {
      nX0 = js.px[jw0 + lane];
      nY0 = js.py[jw0 + lane];
      nZ0 = js.pz[jw0 + lane];
      nV0 = js.vm[jw0 + lane];
    }
    if (jw0 + 32 + lane < jw1) {
      nX1 = js.px[jw0 + 32 + lane];
      nY1 = js.py[jw0 + 32 + lane];
      nZ1 = js.pz[jw0 + 32 + lane];
      nV1 = js.vm[jw0 + 32 + lane];
    }
    // targets, held negated as double-single hi/lo; r2g < 0 marks an unused slot
    float nhx[MI], nhy[MI], nhz[MI], nlx[MI], nly[MI], nlz[MI], nvx[MI], nvy[MI], nvz[MI], r2g[MI];
#pragma unroll
    for (int k = 0; k < MI; ++k) {
      const bool valid = ig + k < w.m;
      const int t = w.order_t[valid ? ig + k : ig];
      const double X = js.px[t], Y = js.py[t], Z = js.pz[t];
      const float fx = (float)X, fy = (float)Y, fz = (float)Z;
      nhx[k] = -fx;
      nhy[k] = -fy;
      nhz[k] = -fz;
      nlx[k] = -(float)(X - (double)fx);
      nly[k] = -(float)(Y - (double)fy);
      nlz[k] = -(float)(Z - (double)fz);
      const float4 vmi = js.vm[t];
      nvx[k] = -vmi.x;
      nvy[k] = -vmi.y;
      nvz[k] = -vmi.z;
      // the tile kernel's candidate threshold with double-single offsets: every
      // FP64 neighbour (r2 < R2) passes r2f < r2g, and so does the self pair
      const double R = sqrt(fmax(js.r2nb[t], 0.0));
      const double Rg = R * (1.0 + 0x1p-17) + 1e-30;
      float g = __double2float_ru(Rg * Rg + w.eps2);
      g = fmaxf(g, nextafterf(w.eps2f, FLT_MAX));
      r2g[k] = valid ? g : -1.0f;
    }
    float2 p[MI][6];
#pragma unroll
    for (int k = 0; k < MI; ++k)
#pragma unroll
      for (int c = 0; c < 6; ++c) p[k][c] = make_float2(0.0f, 0.0f);

    for (int jb = jw0; jb < jw1; jb += 64) {
      const int ja = jb + lane, jc = jb + 32 + lane;
      const bool ina = ja < jw1, inc = jc < jw1;
      const double X0 = nX0, Y0 = nY0, Z0 = nZ0, X1 = nX1, Y1 = nY1, Z1 = nZ1;
      const float4 V0 = nV0, V1 = nV1;
      {
        const int qa = jb + 64 + lane, qc = jb + 96 + lane;
        nX0 = nY0 = nZ0 = nX1 = nY1 = nZ1 = 1e30;
        nV0 = nV1 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (qa < jw1) {
          nX0 = js.px[qa];
          nY0 = js.py[qa];
          nZ0 = js.pz[qa];
          nV0 = js.vm[qa];
        }
        if (qc < jw1) {
          nX1 = js.px[qc];
          nY1 = js.py[qc];
          nZ1 = js.pz[qc];
          nV1 = js.vm[qc];
        }
      }
      const float2 xh = make_float2((float)X0, (float)X1);
      const float2 yh = make_float2((float)Y0, (float)Y1);
      const float2 zh = make_float2((float)Z0, (float)Z1);
      const float2 xl = make_float2((float)(X0 - (double)xh.x), (float)(X1 - (double)xh.y));
      const float2 yl = make_float2((float)(Y0 - (double)yh.x), (float)(Y1 - (double)yh.y));
      const float2 zl = make_float2((float)(Z0 - (double)zh.x), (float)(Z1 - (double)zh.y));
      const float2 vx = make_float2(V0.x, V1.x);
      const float2 vy = make_float2(V0.y, V1.y);
      const float2 vz = make_float2(V0.z, V1.z);
      const float2 mj = make_float2(V0.w, V1.w);
      bool any = false;
#pragma unroll
      for (int k = 0; k < MI; ++k) {
        if (r2g[k] < 0.0f) continue;  // the same for every lane
        const PairGeom2 g = pair_geom2_ds(xh, yh, zh, xl, yl, zl, vx, vy, vz, dup2(nhx[k]), dup2(nhy[k]),
                                          dup2(nhz[k]), dup2(nlx[k]), dup2(nly[k]), dup2(nlz[k]), dup2(nvx[k]),
                                          dup2(nvy[k]), dup2(nvz[k]), eps2v);
        const bool c0 = g.r2.x < r2g[k];
        const bool c1 = g.r2.y < r2g[k];
        float2 ri;
        ri.x = c0 ? 0.0f : rsqrtf(g.r2.x);
        ri.y = c1 ? 0.0f : rsqrtf(g.r2.y);
        any |= (c0 | c1);
        pair_accum2(g, mj, ri, p[k]);
      }
      if (any) {
        // slow path, this lane only: candidates re-decided with the FP64 test
#pragma unroll
        for (int k = 0; k < MI; ++k) {
          if (r2g[k] < 0.0f) continue;
          const PairGeom2 g = pair_geom2_ds(xh, yh, zh, xl, yl, zl, vx, vy, vz, dup2(nhx[k]), dup2(nhy[k]),
                                            dup2(nhz[k]), dup2(nlx[k]), dup2(nly[k]), dup2(nlz[k]),
                                            dup2(nvx[k]), dup2(nvy[k]), dup2(nvz[k]), eps2v);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const float r2f = h ? g.r2.y : g.r2.x;
            if (!(r2f < r2g[k]) || !(h ? inc : ina)) continue;
            const int j = h ? jc : ja;
            const int t = w.order_t[ig + k];
            if (j == t) continue;
            const double r2e = exact_r2(js.px[t], js.py[t], js.pz[t], js.px[j], js.py[j], js.pz[j]);
            if (r2e < js.r2nb[t]) {
              const int row = w.order_o[ig + k];
              const int idx = atomicAdd(&w.lcnt[row], 1);
              if (idx < w.cap) w.lst[(size_t)row * w.cap + idx] = j;
            } else {
              const float rr = rsqrtf(r2f);
              pair_accum2(g, mj, h ? make_float2(0.0f, rr) : make_float2(rr, 0.0f), p[k]);
            }
          }
        }
      }
    }
    // lane halves and lanes in FP64 (fixed tree), then the block's warps in order
#pragma unroll
    for (int k = 0; k < MI; ++k) {
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        double sum = (double)p[k][c].x + (double)p[k][c].y;
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL, sum, o);
        if (lane == 0) s_red[warp][k][c] = sum;
      }
    }
    __syncthreads();
    if (threadIdx.x < MI * 6) {
      const int k = threadIdx.x / 6, c = threadIdx.x - 6 * (threadIdx.x / 6);
      if (ig + k < w.m) {
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < kJmWarps; ++q) sum += s_red[q][k][c];
        w.part[((size_t)w.order_o[ig + k] * w.s_stride + ch) * 6 + c] = sum;
      }
    }
    __syncthreads();
  }
  if (fuse_sort_cap > 0) {
    // the block that finishes last finalizes the rows in place (few rows): no
    // second launch.  Every block's partials and list entries are made visible
    // before it counts itself done; no block waits on another.
    extern __shared__ int fin_smem[];
    __shared__ double red[kJmWarps][6];
    __shared__ int s_nl_total[2];
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(w.item_counter, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (s_last) {
      __threadfence();
      for (int r = 0; r < w.m; ++r) finalize_row_block<32 * kJmWarps>(js, w, o, fuse_sort_cap, r, fin_smem, red,
                                                                       s_nl_total);
    }
  }
}

// ============================================================ list sort
// The row's nl list entries (distinct j) from lrow, sorted ascending into
// buf[0..nl) by the calling threads (tid of nthr), with buf of P >= 2 nl ints:
// entry k is staged at buf[P/2 + k] and placed at its rank, the number of
// entries smaller than it.  `sync` orders the staging before the ranking.
template <class Sync>
__device__ __forceinline__ void rank_sort(const int *lrow, int nl, int *buf, int P, int tid, int nthr, Sync sync) {
  int *stage = buf + P / 2;
  // L2-coherent: the entries may come from other blocks of the same launch
  for (int k = tid; k < nl; k += nthr) stage[k] = __ldcg(&lrow[k]);
  sync();
  for (int k = tid; k < nl; k += nthr) {
    const int e = stage[k];
    int rank = 0;
    for (int q = 0; q < nl; ++q) rank += stage[q] < e;
    buf[rank] = e;
  }
  sync();
}

__device__ void relist_row(const JSet &js, const Work &w, const Outputs &o, int r);

// ============================================================ finalize
// One warp per output row.  Regular part: FP64 sum of the chunk partials in a
// fixed lane/tree order.  List: the row's entries (appended by chunks in any
// order) are sorted ascending with a warp bitonic sort in shared memory.
// Irregular part: the reference's FP64 formula (ComputeAcceleration.cpp:
// 285-292, softened as for the regular part) over the final list, lane-strided
// with a fixed reduction tree.
__global__ void finalize_rows(JSet js, Work w, Outputs o, int sort_cap) {
  extern __shared__ int fin_smem[];
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int *buf = fin_smem + (threadIdx.x >> 5) * sort_cap;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int m_rows = w.m_dev ? *w.m_dev : w.m;
  for (int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < m_rows; r += nwarps) {
    double s[6] = {0, 0, 0, 0, 0, 0};
    const int nch = w.row_nchunks ? w.row_nchunks[r] : w.n_chunks;
    const int joff = w.row_joff ? w.row_joff[r] : 0;
    // unrolled so that the loads of several chunks are in flight at once; the
    // additions keep their order (chunk c, c + 32, ...), so the sum is unchanged
#pragma unroll 8
    for (int c = lane; c < nch; c += 32) {
      const double *src = w.part + ((size_t)r * w.s_stride + c) * 6;
#pragma unroll
      for (int q = 0; q < 6; ++q) s[q] += src[q];
    }
#pragma unroll
    for (int q = 0; q < 6; ++q)
      for (int off = 16; off > 0; off >>= 1) s[q] += __shfl_xor_sync(FULL, s[q], off);

    const int total = w.lcnt[r];
    const int nl = min(total, w.cap);
    int *lrow = w.lst + (size_t)r * w.cap;
    int *out = o.list + (size_t)r * w.cap;
    // short lists (most): rank sort; longer ones: bitonic sort of nl
    // entries, padded to a power of two >= 32
    const bool by_rank = 2 * nl <= sort_cap;
    if (by_rank) rank_sort(lrow, nl, buf, sort_cap, lane, 32, []() { __syncwarp(); });
    int P = 32;
    while (P < nl) P <<= 1;
    if (!by_rank)
      for (int k = lane; k < P; k += 32) buf[k] = k < nl ? lrow[k] : INT_MAX;
    __syncwarp();
    for (int kk = 2; kk <= (by_rank ? 1 : P); kk <<= 1) {
      for (int jj = kk >> 1; jj > 0; jj >>= 1) {
        for (int i = lane; i < P; i += 32) {
          const int l = i ^ jj;
          if (l > i) {
            const int a = buf[i], b = buf[l];
            const bool up = (i & kk) == 0;
            if ((a > b) == up) {
              buf[i] = b;
              buf[l] = a;
            }
          }
        }
        __syncwarp();
      }
    }
    for (int k = lane; k < nl; k += 32) out[k] = buf[k] - joff;
    __syncwarp();

    const int t = o.targets[r];
    const double xi = js.px[t], yi = js.py[t], zi = js.pz[t];
    const double vxi = js.pvx[t], vyi = js.pvy[t], vzi = js.pvz[t];
    double a[6] = {0, 0, 0, 0, 0, 0};
    for (int k = lane; k < nl; k += 32) {
      const int j = buf[k];
      const double x[3] = {__dsub_rn(js.px[j], xi), __dsub_rn(js.py[j], yi), __dsub_rn(js.pz[j], zi)};
      const double v[3] = {__dsub_rn(js.pvx[j], vxi), __dsub_rn(js.pvy[j], vyi),
                           __dsub_rn(js.pvz[j], vzi)};
      double r2 = 0.0, vx = 0.0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        r2 = __dadd_rn(r2, __dmul_rn(x[d], x[d]));
        vx = __dadd_rn(vx, __dmul_rn(v[d], x[d]));
      }
      const double r2s = __dadd_rn(r2, w.eps2);
      const double m_r3 = __ddiv_rn(__ddiv_rn(js.mass[j], r2s), __dsqrt_rn(r2s));
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        a[d] = __dadd_rn(a[d], __dmul_rn(m_r3, x[d]));
        const double corr = __ddiv_rn(__dmul_rn(__dmul_rn(3.0, x[d]), vx), r2s);
        a[3 + d] = __dadd_rn(a[3 + d], __dmul_rn(m_r3, __dsub_rn(v[d], corr)));
      }
    }
#pragma unroll
    for (int q = 0; q < 6; ++q)
      for (int off = 16; off > 0; off >>= 1) a[q] += __shfl_xor_sync(FULL, a[q], off);

    if (lane == 0) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        o.acc_reg[3 * r + d] = s[d];
        o.jerk_reg[3 * r + d] = s[3 + d];
        o.acc_irr[3 * r + d] = a[d];
        o.jerk_irr[3 * r + d] = a[3 + d];
      }
      o.nnb[r] = total;
      if (total > w.cap) {
        const int q = atomicAdd(o.overflow_rows, 1);
        o.ovf_list[q] = r;
        atomicOr(w.status, kErrOverflow);
      }
    }
    __syncwarp();
  }
}

// One block per output row, for launches with few rows (the warp-per-row
// kernel above leaves most of the GPU idle there and is latency-bound).  The
// same three parts: the chunk partials summed by every thread (thread t adds
// chunks t, t + NT, ... in order, then the thread sums are added in a fixed
// tree), the list sorted by warp 0 as above, and the irregular part with one
// neighbour per thread, added in a fixed tree.
template <int NT>
__device__ __forceinline__ void block_sum6(double (&v)[6], double (*red)[6]) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 6; ++q)
    for (int off = 16; off > 0; off >>= 1) v[q] += __shfl_xor_sync(FULL, v[q], off);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 6; ++q) red[warp][q] = v[q];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      double t = 0.0;
      for (int k = 0; k < NT / 32; ++k) t += red[k][q];
      v[q] = t;
    }
  __syncthreads();
}

// One row's finalize by a block of NT threads (called by every thread of the
// block): FP64 sum of the chunk partials, the sorted list, the FP64 irregular
// part, and the re-list of an overflowed row.  Reads that may see other
// blocks' writes of the same launch are L2-coherent, so the force kernel's last
// block can finalize in place (reg_force_jmajor with fused rows).
template <int NT>
__device__ void finalize_row_block(const JSet &js, const Work &w, const Outputs &o, int sort_cap, int r,
                                   int *fin_smem, double (*red)[6], int *s_nl_total) {
  const int nch = w.row_nchunks ? w.row_nchunks[r] : w.n_chunks;
  const int joff = w.row_joff ? w.row_joff[r] : 0;
  // chunk partials: thread g * 6 + q adds component q of chunks g, g + G, ...
  // into eight sums by turn (eight independent loads in flight), which it adds
  // in order; then the G sums of a component are added in g order
  constexpr int G = NT / 6;
  constexpr int A = 8;
  __shared__ double s_part[G * 6];
  if (threadIdx.x < G * 6) {
    const int g = threadIdx.x / 6, q = threadIdx.x - 6 * g;
    const double *src = w.part + (size_t)r * w.s_stride * 6 + q;
    double acc[A];
#pragma unroll
    for (int k = 0; k < A; ++k) acc[k] = 0.0;
    int c = g;
    for (; c + (A - 1) * G < nch; c += A * G) {
      double v[A];
#pragma unroll
      for (int k = 0; k < A; ++k) v[k] = __ldcg(&src[(size_t)(c + k * G) * 6]);
#pragma unroll
      for (int k = 0; k < A; ++k) acc[k] += v[k];
    }
#pragma unroll
    for (int k = 0; k < A; ++k)
      if (c + k * G < nch) acc[k] += __ldcg(&src[(size_t)(c + k * G) * 6]);
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < A; ++k) t += acc[k];
    s_part[threadIdx.x] = t;
  }
  __syncthreads();
  double s[6] = {0, 0, 0, 0, 0, 0};
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      double t = 0.0;
      for (int g = 0; g < G; ++g) t += s_part[6 * g + q];
      s[q] = t;
    }

  {
    const int total = __ldcg(&w.lcnt[r]);
    const int nl = min(total, w.cap);
    if (threadIdx.x == 0) {
      s_nl_total[0] = nl;
      s_nl_total[1] = total;
    }
    if (2 * nl <= sort_cap)
      rank_sort(w.lst + (size_t)r * w.cap, nl, fin_smem, sort_cap, threadIdx.x, NT, []() { __syncthreads(); });
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 32 && 2 * s_nl_total[0] > sort_cap) {
    const int nl = s_nl_total[0];
    const int *lrow = w.lst + (size_t)r * w.cap;
    int P = 32;
    while (P < nl) P <<= 1;
    int *buf = fin_smem;
    for (int k = lane; k < P; k += 32) buf[k] = k < nl ? __ldcg(&lrow[k]) : INT_MAX;
    __syncwarp();
    for (int kk = 2; kk <= P; kk <<= 1) {
      for (int jj = kk >> 1; jj > 0; jj >>= 1) {
        for (int i = lane; i < P; i += 32) {
          const int l = i ^ jj;
          if (l > i) {
            const int a = buf[i], b = buf[l];
            const bool up = (i & kk) == 0;
            if ((a > b) == up) {
              buf[i] = b;
              buf[l] = a;
            }
          }
        }
        __syncwarp();
      }
    }
  }
  __syncthreads();
  const int nl = s_nl_total[0], total = s_nl_total[1];
  const int *buf = fin_smem;
  int *out = o.list + (size_t)r * w.cap;
  for (int k = threadIdx.x; k < nl; k += NT) out[k] = buf[k] - joff;

  const int t = o.targets[r];
  const double xi = js.px[t], yi = js.py[t], zi = js.pz[t];
  const double vxi = js.pvx[t], vyi = js.pvy[t], vzi = js.pvz[t];
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int k = threadIdx.x; k < nl; k += NT) {
    const int j = buf[k];
    const double x[3] = {__dsub_rn(js.px[j], xi), __dsub_rn(js.py[j], yi), __dsub_rn(js.pz[j], zi)};
    const double v[3] = {__dsub_rn(js.pvx[j], vxi), __dsub_rn(js.pvy[j], vyi), __dsub_rn(js.pvz[j], vzi)};
    double r2 = 0.0, vx = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      r2 = __dadd_rn(r2, __dmul_rn(x[d], x[d]));
      vx = __dadd_rn(vx, __dmul_rn(v[d], x[d]));
    }
    const double r2s = __dadd_rn(r2, w.eps2);
    const double m_r3 = __ddiv_rn(__ddiv_rn(js.mass[j], r2s), __dsqrt_rn(r2s));
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      a[d] = __dadd_rn(a[d], __dmul_rn(m_r3, x[d]));
      const double corr = __ddiv_rn(__dmul_rn(__dmul_rn(3.0, x[d]), vx), r2s);
      a[3 + d] = __dadd_rn(a[3 + d], __dmul_rn(m_r3, __dsub_rn(v[d], corr)));
    }
  }
  block_sum6<NT>(a, red);

  if (threadIdx.x == 0) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      o.acc_reg[3 * r + d] = s[d];
      o.jerk_reg[3 * r + d] = s[3 + d];
      o.acc_irr[3 * r + d] = a[d];
      o.jerk_irr[3 * r + d] = a[3 + d];
    }
    o.nnb[r] = total;
    if (total > w.cap) {
      const int q = atomicAdd(o.overflow_rows, 1);
      o.ovf_list[q] = r;
      atomicOr(w.status, kErrOverflow);
    }
  }
  __syncthreads();
  // an overflowed row is re-listed here, by warp 0, instead of by relist_rows
  if (total > w.cap && threadIdx.x < 32) relist_row(js, w, o, r);
  __syncthreads();
}

template <int NT>
__global__ void __launch_bounds__(NT) finalize_rows_block(JSet js, Work w, Outputs o, int sort_cap) {
  extern __shared__ int fin_smem[];  // the row's sort buffer
  __shared__ double red[NT / 32][6];
  __shared__ int s_nl_total[2];
  const int m_rows = w.m_dev ? *w.m_dev : w.m;
  for (int r = blockIdx.x; r < m_rows; r += gridDim.x)
    finalize_row_block<NT>(js, w, o, sort_cap, r, fin_smem, red, s_nl_total);
}

// ============================================================ re-list
// Rows whose neighbours did not fit in cap were appended in chunk order and kept
// an arbitrary subset.  One warp per such row scans the row's j-range in
// ascending order with the exact FP64 test, keeps the first cap neighbours
// (ballot + popc placement) and recomputes the irregular part over all of them,
// so an overflowed row reads like the reference's truncated CPU list.
// One warp re-lists row r (see above).
__device__ void relist_row(const JSet &js, const Work &w, const Outputs &o, int r) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;
  const int t = o.targets[r];
  const int joff = w.row_joff ? w.row_joff[r] : 0;
  const int j1 = joff + (w.row_jlen ? w.row_jlen[r] : js.n);
  const double xi = js.px[t], yi = js.py[t], zi = js.pz[t];
  const double vxi = js.pvx[t], vyi = js.pvy[t], vzi = js.pvz[t];
  const double R2 = js.r2nb[t];
  int *out = o.list + (size_t)r * w.cap;
  int base = 0;
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int jb = joff; jb < j1; jb += 32) {
    const int j = jb + lane;
    bool isnb = false;
    double x[3] = {0, 0, 0}, r2 = 0.0;
    if (j < j1 && j != t) {
      x[0] = __dsub_rn(js.px[j], xi);
      x[1] = __dsub_rn(js.py[j], yi);
      x[2] = __dsub_rn(js.pz[j], zi);
      r2 = __dmul_rn(x[0], x[0]);
      r2 = __dadd_rn(r2, __dmul_rn(x[1], x[1]));
      r2 = __dadd_rn(r2, __dmul_rn(x[2], x[2]));
      isnb = r2 < R2;
    }
    const unsigned mask = __ballot_sync(FULL, isnb);
    if (isnb) {
      const int pos = base + __popc(mask & lt_mask);
      if (pos < w.cap) out[pos] = j - joff;
      const double v[3] = {__dsub_rn(js.pvx[j], vxi), __dsub_rn(js.pvy[j], vyi), __dsub_rn(js.pvz[j], vzi)};
      double vx = 0.0;
#pragma unroll
      for (int d = 0; d < 3; ++d) vx = __dadd_rn(vx, __dmul_rn(v[d], x[d]));
      const double r2s = __dadd_rn(r2, w.eps2);
      const double m_r3 = __ddiv_rn(__ddiv_rn(js.mass[j], r2s), __dsqrt_rn(r2s));
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        a[d] = __dadd_rn(a[d], __dmul_rn(m_r3, x[d]));
        const double corr = __ddiv_rn(__dmul_rn(__dmul_rn(3.0, x[d]), vx), r2s);
        a[3 + d] = __dadd_rn(a[3 + d], __dmul_rn(m_r3, __dsub_rn(v[d], corr)));
      }
    }
    base += __popc(mask);
  }
#pragma unroll
  for (int k = 0; k < 6; ++k)
    for (int off = 16; off > 0; off >>= 1) a[k] += __shfl_xor_sync(FULL, a[k], off);
  if (lane == 0) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      o.acc_irr[3 * r + d] = a[d];
      o.jerk_irr[3 * r + d] = a[3 + d];
    }
  }
}

__global__ void relist_rows(JSet js, Work w, Outputs o) {
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int nrows = *o.overflow_rows;
  for (int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < nrows; q += nwarps) relist_row(js, w, o, o.ovf_list[q]);
}

// ============================================================ energy
// FP64 kinetic + softened potential energy; one block of 256 threads per i-tile
// of 256, j looped; per-i potentials written for a deterministic host sum.
__global__ void energy_rows(int n, const double *__restrict__ x, const double *__restrict__ v,
                            const double *__restrict__ mass, double eps2,
                            double *__restrict__ e_row) {
  __shared__ double sx[256], sy[256], sz[256], sm[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double xi = 0, yi = 0, zi = 0;
  if (i < n) {
    xi = x[3 * i];
    yi = x[3 * i + 1];
    zi = x[3 * i + 2];
  }
  double w = 0.0;
  for (int jt = 0; jt < n; jt += 256) {
    const int j = jt + threadIdx.x;
    __syncthreads();
    if (j < n) {
      sx[threadIdx.x] = x[3 * j];
      sy[threadIdx.x] = x[3 * j + 1];
      sz[threadIdx.x] = x[3 * j + 2];
      sm[threadIdx.x] = mass[j];
    } else {
      sx[threadIdx.x] = sy[threadIdx.x] = sz[threadIdx.x] = 0.0;
      sm[threadIdx.x] = 0.0;
    }
    __syncthreads();
    const int lim = min(256, n - jt);
    for (int jj = 0; jj < lim; ++jj) {
      if (jt + jj == i) continue;
      const double dx = sx[jj] - xi, dy = sy[jj] - yi, dz = sz[jj] - zi;
      const double r2 = dx * dx + dy * dy + dz * dz + eps2;
      w += sm[jj] * rsqrt(r2);
    }
  }
  if (i < n) {
    const double v2 = v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2];
    e_row[i] = 0.5 * mass[i] * v2 - 0.5 * mass[i] * w;
  }
}

// ============================================================ launch wrappers
void launch_predict(cudaStream_t s, int n, const double *x, const double *v, const double *a0,
                    const double *a1, const double *t0, const double *mass, double new_time,
                    double time_scale, double *px, double *py, double *pz, double *pvx,
                    double *pvy, double *pvz, float4 *vm, int sm_count) {
  const int blocks = min((n + 255) / 256, sm_count * 8);
  predict_jset<<<max(blocks, 1), 256, 0, s>>>(n, x, v, a0, a1, t0, mass, new_time, time_scale, px, py,
                                               pz, pvx, pvy, pvz, vm);
}

void launch_pack_vm(cudaStream_t s, int n, const double *pvx, const double *pvy, const double *pvz,
                    const double *mass, float4 *vm, int sm_count) {
  const int blocks = min((n + 255) / 256, sm_count * 8);
  pack_vm<<<max(blocks, 1), 256, 0, s>>>(n, pvx, pvy, pvz, mass, vm);
}

void launch_unpack_predicted(cudaStream_t s, int n, const double *pos, const double *vel,
                             const double *mass, double *px, double *py, double *pz, double *pvx,
                             double *pvy, double *pvz, float4 *vm, int sm_count) {
  const int blocks = min((n + 255) / 256, sm_count * 8);
  unpack_predicted<<<max(blocks, 1), 256, 0, s>>>(n, pos, vel, mass, px, py, pz, pvx, pvy, pvz, vm);
}

void launch_iota(cudaStream_t s, int m, int *out, int sm_count) {
  iota_kernel<<<max(1, min((m + 255) / 256, sm_count * 8)), 256, 0, s>>>(m, out);
}

size_t sort_temp_bytes(int m_cap) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint32_t *)nullptr, (uint32_t *)nullptr,
                                  (const int *)nullptr, (int *)nullptr, m_cap, 0, 30);
  return bytes;
}

void launch_spatial_order(cudaStream_t s, int m, const int *targets, const JSet &js, int *bbox,
                          uint32_t *keys, uint32_t *keys_alt, int *rows, int *rows_alt, void *cub_tmp,
                          size_t cub_bytes, int *order_t, int *order_o, int per_block, double *anchor,
                          int sm_count) {
  const int init[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
  cudaMemcpyAsync(bbox, init, sizeof(init), cudaMemcpyHostToDevice, s);
  const int blocks = max(1, min((m + 255) / 256, sm_count * 4));
  target_bbox<<<blocks, 256, 0, s>>>(m, targets, js.px, js.py, js.pz, bbox);
  target_curve_key<<<blocks, 256, 0, s>>>(m, targets, js.px, js.py, js.pz, bbox, keys, rows);
  size_t bytes = cub_bytes;
  cub::DeviceRadixSort::SortPairs(cub_tmp, bytes, keys, keys_alt, rows, rows_alt, m, 0, 30, s);
  gather_order<<<blocks, 256, 0, s>>>(m, targets, rows_alt, order_t, order_o);
  if (anchor) {
    const int nblk = (m + per_block - 1) / per_block;
    const int ablocks = max(1, min((nblk + 7) / 8, sm_count * 4));
    block_anchor<<<ablocks, 256, 0, s>>>(m, per_block, order_t, js.px, js.py, js.pz, anchor);
  }
}

// ------------------------------------------------------------------ tile variants
// Each instantiated shape of reg_force_tile: (threads, targets per thread,
// anchor/double-single offsets, packed FP32x2 arithmetic, j unroll, minimum
// resident CTAs per SM as a register cap).
struct TileVariant {
  int nt, ipt, anchor, pack, unr, minb;
  int (*occupancy)();
  void (*launch)(cudaStream_t, int, const JSet &, const Work &, int);
};

template <int NT, int IPT, bool ANCHOR, bool PACK, int UNR, int MINB>
static int tile_occ() {
  constexpr int TJ = 128, NST = 3;
  auto k = reg_force_tile<NT, IPT, TJ, NST, ANCHOR, PACK, UNR, MINB>;
  const size_t sm = TileLayout<NT, IPT, TJ, NST, ANCHOR, PACK>::bytes;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  int blocks = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, NT, sm);
  return blocks;
}

template <int NT, int IPT, bool ANCHOR, bool PACK, int UNR, int MINB>
static void tile_run(cudaStream_t s, int grid, const JSet &js, const Work &w, int n_iblocks) {
  constexpr int TJ = 128, NST = 3;
  auto k = reg_force_tile<NT, IPT, TJ, NST, ANCHOR, PACK, UNR, MINB>;
  const size_t sm = TileLayout<NT, IPT, TJ, NST, ANCHOR, PACK>::bytes;
  k<<<grid, NT, sm, s>>>(js, w, n_iblocks);
}

#define TV(NT, IPT, A, P, U, M) \
  {NT, IPT, A, P, U, M, &tile_occ<NT, IPT, A, P, U, M>, &tile_run<NT, IPT, A, P, U, M>}
#define TV2(NT, IPT, P, U, M) TV(NT, IPT, true, P, U, M), TV(NT, IPT, false, P, U, M)

static const TileVariant kTileVariants[] = {
    // scalar pair arithmetic
    TV2(32, 1, false, 2, 1), TV2(64, 1, false, 2, 1), TV2(128, 1, false, 2, 1), TV2(128, 2, false, 2, 1),
    TV2(128, 4, false, 2, 1), TV2(256, 2, false, 2, 1),
    // packed FP32x2 pair arithmetic (odd ipt: the last target of a thread on scalar arithmetic)
    TV2(128, 2, true, 2, 1), TV2(128, 2, true, 2, 4), TV2(128, 4, true, 1, 1), TV2(128, 4, true, 2, 1),
    TV2(128, 4, true, 2, 3), TV2(128, 4, true, 1, 4), TV2(256, 2, true, 2, 1), TV2(256, 4, true, 1, 2),
    TV2(256, 4, true, 2, 1), TV2(128, 2, true, 1, 5), TV2(128, 2, true, 4, 4), TV2(128, 4, true, 2, 4),
    TV2(256, 4, true, 2, 2), TV2(128, 8, true, 1, 2), TV2(128, 6, true, 1, 2), TV2(128, 3, true, 2, 4), TV(128, 6, true, true, 1, 3),
};
#undef TV2
#undef TV

// First variant matching the request; unroll/min_blocks of 0 match anything.
static const TileVariant *find_variant(int nt, int ipt, bool anchor, bool pack, int unr, int minb) {
  for (const TileVariant &v : kTileVariants)
    if (v.nt == nt && v.ipt == ipt && v.anchor == (int)anchor && v.pack == (int)pack &&
        (unr == 0 || v.unr == unr) && (minb == 0 || v.minb == minb))
      return &v;
  return nullptr;
}

int tile_occupancy(int nt, int ipt, bool anchor, bool pack, int unr, int minb) {
  const TileVariant *v = find_variant(nt, ipt, anchor, pack, unr, minb);
  if (!v) return -1;
  const int occ = v->occupancy();
  // the dynamic smem attribute is set on the first query; check it stuck
  return cudaGetLastError() == cudaSuccess ? occ : -1;
}

int launch_tile(cudaStream_t s, int nt, int ipt, bool anchor, bool pack, int unr, int minb, int grid,
                const JSet &js, const Work &w, int n_iblocks) {
  const TileVariant *v = find_variant(nt, ipt, anchor, pack, unr, minb);
  if (!v) return -1;
  v->launch(s, grid, js, w, n_iblocks);
  return 0;
}

// Warps sharing targets: 4 warps, double-single offsets, 32 x ipt targets per
// block.  Kernel 4: scalar pair arithmetic, 1 or 2 j per step.  Kernel 5
// (packed): FP32x2 over the two targets of a thread (ipt 2, 1 or 2 j per
// step) or over two j (ipt 1).
template <int IPT, int UNR, bool PK>
static int split_occ() {
  constexpr int TJ = 128, NST = 3, NT = 128;
  constexpr bool PACK = PK && IPT == 2, PJ = PK && IPT == 1;
  auto k = reg_force_tile<NT, IPT, TJ, NST, false, PACK, UNR, 1, 4, PJ>;
  const size_t sm = TileLayout<NT, IPT, TJ, NST, false, PACK>::bytes;
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  int blocks = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, NT, sm);
  return blocks;
}

template <int IPT, int UNR, bool PK>
static void split_run(cudaStream_t s, int grid, const JSet &js, const Work &w, int n_iblocks) {
  constexpr int TJ = 128, NST = 3, NT = 128;
  constexpr bool PACK = PK && IPT == 2, PJ = PK && IPT == 1;
  auto k = reg_force_tile<NT, IPT, TJ, NST, false, PACK, UNR, 1, 4, PJ>;
  const size_t sm = TileLayout<NT, IPT, TJ, NST, false, PACK>::bytes;
  k<<<grid, NT, sm, s>>>(js, w, n_iblocks);
}

int tile_split_occupancy(int ipt, int unr, bool packed) {
  int occ = -1;
  if (!packed && ipt == 1) occ = unr == 2 ? split_occ<1, 2, false>() : split_occ<1, 1, false>();
  if (!packed && ipt == 2) occ = unr == 2 ? split_occ<2, 2, false>() : split_occ<2, 1, false>();
  if (packed && ipt == 1) occ = split_occ<1, 1, true>();
  if (packed && ipt == 2) occ = unr == 2 ? split_occ<2, 2, true>() : split_occ<2, 1, true>();
  return cudaGetLastError() == cudaSuccess ? occ : -1;
}

int launch_tile_split(cudaStream_t s, int ipt, int unr, bool packed, int grid, const JSet &js, const Work &w,
                      int n_iblocks) {
  if (!packed && ipt == 1 && unr == 2)
    split_run<1, 2, false>(s, grid, js, w, n_iblocks);
  else if (!packed && ipt == 1 && unr == 1)
    split_run<1, 1, false>(s, grid, js, w, n_iblocks);
  else if (!packed && ipt == 2 && unr == 2)
    split_run<2, 2, false>(s, grid, js, w, n_iblocks);
  else if (!packed && ipt == 2 && unr == 1)
    split_run<2, 1, false>(s, grid, js, w, n_iblocks);
  else if (packed && ipt == 1)
    split_run<1, 1, true>(s, grid, js, w, n_iblocks);
  else if (packed && ipt == 2 && unr == 2)
    split_run<2, 2, true>(s, grid, js, w, n_iblocks);
  else if (packed && ipt == 2 && unr == 1)
    split_run<2, 1, true>(s, grid, js, w, n_iblocks);
  else
    return -1;
  return 0;
}

int tile_variant_count() { return (int)(sizeof(kTileVariants) / sizeof(kTileVariants[0])); }

int tile_variant_shape(int i, int *shape6) {
  if (i < 0 || i >= tile_variant_count()) return -1;
  const TileVariant &v = kTileVariants[i];
  shape6[0] = v.nt;
  shape6[1] = v.ipt;
  shape6[2] = v.anchor;
  shape6[3] = v.pack;
  shape6[4] = v.unr;
  shape6[5] = v.minb;
  return 0;
}

int jmajor_warps() { return kJmWarps; }

int jmajor_occupancy(int mi) {
  int occ = 0;
  cudaError_t e = cudaErrorInvalidValue;
  switch (mi) {
    case 1: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, reg_force_jmajor<1>, 32 * kJmWarps, 0); break;
    case 2: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, reg_force_jmajor<2>, 32 * kJmWarps, 0); break;
    case 4: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, reg_force_jmajor<4>, 32 * kJmWarps, 0); break;
    case 8: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, reg_force_jmajor<8>, 32 * kJmWarps, 0); break;
    default: break;
  }
  return e == cudaSuccess ? std::max(occ, 1) : 1;
}

int launch_jmajor(cudaStream_t s, int mi, const JSet &js, const Work &w, int Lw, const Outputs *fuse) {
  // one block per j-chunk (w.n_chunks of them), kJmWarps sub-chunks of Lw each;
  // with `fuse`, the last block to finish finalizes the rows (w.item_counter
  // must be zero)
  const int blocks = w.n_chunks;
  int P = 0;
  size_t smem = 0;
  Outputs o{};
  if (fuse) {
    o = *fuse;
    P = 32;
    while (P < w.cap) P <<= 1;
    smem = (size_t)P * sizeof(int);
  }
  auto go = [&](auto kern) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kern<<<blocks, 32 * kJmWarps, smem, s>>>(js, w, o, Lw, P);
  };
  switch (mi) {
    case 1: go(reg_force_jmajor<1>); break;
    case 2: go(reg_force_jmajor<2>); break;
    case 4: go(reg_force_jmajor<4>); break;
    case 8: go(reg_force_jmajor<8>); break;
    default: return -1;
  }
  return 0;
}

void launch_finalize(cudaStream_t s, const JSet &js, const Work &w, const Outputs &o, int sm_count) {
  int P = 32;
  while (P < w.cap) P <<= 1;
  if (w.m <= 2 * sm_count) {
    // few rows: a block per row
    const size_t smem = (size_t)P * sizeof(int);
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(finalize_rows_block<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    finalize_rows_block<128><<<w.m, 128, smem, s>>>(js, w, o, P);
    return;
  }
  const int warps_per_block = 4;
  const size_t smem = (size_t)warps_per_block * P * sizeof(int);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(finalize_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int blocks = max(1, min((w.m + warps_per_block - 1) / warps_per_block, sm_count * 32));
  finalize_rows<<<blocks, 32 * warps_per_block, smem, s>>>(js, w, o, P);
  relist_rows<<<sm_count * 4, 128, 0, s>>>(js, w, o);
}

void launch_predict_multi(cudaStream_t s, int n, const int *cid, const int *active,
                          const double *new_time, const double *time_scale, const double *x,
                          const double *v, const double *a0, const double *a1, const double *t0,
                          const double *mass, double *px, double *py, double *pz, double *pvx,
                          double *pvy, double *pvz, float4 *vm, int sm_count) {
  const int blocks = max(1, min((n + 255) / 256, sm_count * 8));
  predict_multi<<<blocks, 256, 0, s>>>(n, cid, active, new_time, time_scale, x, v, a0, a1, t0, mass, px,
                                       py, pz, pvx, pvy, pvz, vm);
}

void launch_finalize_grid(cudaStream_t s, const JSet &js, const Work &w, const Outputs &o, int blocks) {
  int P = 32;
  while (P < w.cap) P <<= 1;
  const size_t smem = (size_t)4 * P * sizeof(int);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(finalize_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  finalize_rows<<<blocks, 128, smem, s>>>(js, w, o, P);
  relist_rows<<<blocks, 128, 0, s>>>(js, w, o);
}

void launch_energy(cudaStream_t s, int n, const double *x, const double *v, const double *mass,
                   double eps2, double *e_row) {
  energy_rows<<<(n + 255) / 256, 256, 0, s>>>(n, x, v, mass, eps2, e_row);
}

}  // namespace abyss
