// Second and third time derivatives of the acceleration at a common time, the
// initialisation pass of the Ahmad-Cohen scheme (CalculateAcceleration23,
// src_mpi/Particle/Initialize.cpp:102-185), split into a regular part
// (r^2 >= R^2, unsoftened) and an irregular part, with eps2 added to r^2 in the
// force terms.
//
// One thread owns one target and sums its j in ascending order, with every
// operation in the reference's order and rounded to nearest (__dadd_rn etc.;
// this file is also compiled with -fmad=false), so each result equals the
// sequential FP64 host loop bit for bit.  j-particles are staged through
// shared memory in tiles that every thread of the block reads.  The pass is
// O(N^2) with about 25 FP64 divisions per pair; on the host it dominated the
// set-up of every integration.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace abyss {

namespace {

constexpr int kInitThreads = 64;
constexpr int kInitTile = 128;

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// in: x, v, a0 (acc), a1 (jerk) as [n][3]; mass, r2nb [n].  out: [n][12] =
// (reg2, reg3, irr2, irr3) x 3 dimensions.
__global__ void __launch_bounds__(kInitThreads) init_derivs23_kernel(int n, const double *__restrict__ x,
                                                                     const double *__restrict__ v,
                                                                     const double *__restrict__ a0,
                                                                     const double *__restrict__ a1,
                                                                     const double *__restrict__ mass,
                                                                     const double *__restrict__ r2nb,
                                                                     double eps2, double *__restrict__ out) {
  __shared__ double sx[3][kInitTile], sv[3][kInitTile], sa[3][kInitTile], sd[3][kInitTile], sm[kInitTile];
  const int i = blockIdx.x * kInitThreads + threadIdx.x;
  const bool valid = i < n;
  const int ii = valid ? i : 0;
  double xi[3], vi[3], a1i[3], a1doti[3];
  for (int d = 0; d < 3; ++d) {
    xi[d] = x[3 * ii + d];
    vi[d] = v[3 * ii + d];
    a1i[d] = a0[3 * ii + d];
    a1doti[d] = a1[3 * ii + d];
  }
  const double R2 = r2nb[ii];
  double reg2[3] = {0, 0, 0}, reg3[3] = {0, 0, 0}, irr2[3] = {0, 0, 0}, irr3[3] = {0, 0, 0};

  for (int j0 = 0; j0 < n; j0 += kInitTile) {
    const int cnt = min(kInitTile, n - j0);
    __syncthreads();
    for (int t = threadIdx.x; t < cnt; t += kInitThreads) {
      const int j = j0 + t;
      for (int d = 0; d < 3; ++d) {
        sx[d][t] = x[3 * j + d];
        sv[d][t] = v[3 * j + d];
        sa[d][t] = a0[3 * j + d];
        sd[d][t] = a1[3 * j + d];
      }
      sm[t] = mass[j];
    }
    __syncthreads();
    if (!valid) continue;
    for (int t = 0; t < cnt; ++t) {
      if (j0 + t == i) continue;
      double xx[3], vv[3], a21[3], a21dot[3];
      double r2u = 0.0, vr = 0.0, v2 = 0.0, rdf_r2 = 0.0, vdf_r2 = 0.0, rdfdot_r2 = 0.0;
      for (int d = 0; d < 3; ++d) {
        xx[d] = dsub(sx[d][t], xi[d]);
        vv[d] = dsub(sv[d][t], vi[d]);
        r2u = dadd(r2u, dmul(xx[d], xx[d]));
        vr = dadd(vr, dmul(vv[d], xx[d]));
        v2 = dadd(v2, dmul(vv[d], vv[d]));
      }
      const double r2 = dadd(r2u, eps2);
      const double r3 = dmul(r2, __dsqrt_rn(r2));
      const double mj = sm[t];
      const double m_r3 = ddiv(mj, r3);
      for (int d = 0; d < 3; ++d) {
        const double da = dsub(a1i[d], sa[d][t]);
        const double dd = dsub(a1doti[d], sd[d][t]);
        a21[d] = dmul(m_r3, xx[d]);
        // m_r3 * (v - 3 * x * vr / r2)
        a21dot[d] = dmul(m_r3, dsub(vv[d], ddiv(dmul(dmul(3.0, xx[d]), vr), r2)));
        rdf_r2 = dadd(rdf_r2, ddiv(dmul(xx[d], da), r2));
        vdf_r2 = dadd(vdf_r2, ddiv(dmul(vv[d], da), r2));
        rdfdot_r2 = dadd(rdfdot_r2, ddiv(dmul(xx[d], dd), r2));
      }
      const double a = ddiv(vr, r2);
      // b = v2 / r2 + rdf_r2 + a * a
      const double b = dadd(dadd(ddiv(v2, r2), rdf_r2), dmul(a, a));
      // c = 3 * vdf_r2 + rdfdot_r2 + a * (3 * b - 4 * a * a)
      const double c = dadd(dadd(dmul(3.0, vdf_r2), rdfdot_r2), dmul(a, dsub(dmul(3.0, b), dmul(dmul(4.0, a), a))));
      const bool reg = !(r2u < R2);
      for (int d = 0; d < 3; ++d) {
        const double da = dsub(a1i[d], sa[d][t]);
        const double dd = dsub(a1doti[d], sd[d][t]);
        // adot2 = -m * da / r3 - 6 * a * a21dot - 3 * b * a21
        const double adot2 =
            dsub(dsub(ddiv(dmul(-mj, da), r3), dmul(dmul(6.0, a), a21dot[d])), dmul(dmul(3.0, b), a21[d]));
        // adot3 = -m * dd / r3 - 9 * a * adot2 - 9 * b * a21dot - 3 * c * a21
        const double adot3 = dsub(dsub(dsub(ddiv(dmul(-mj, dd), r3), dmul(dmul(9.0, a), adot2)),
                                       dmul(dmul(9.0, b), a21dot[d])),
                                  dmul(dmul(3.0, c), a21[d]));
        if (reg) {
          reg2[d] = dadd(reg2[d], adot2);
          reg3[d] = dadd(reg3[d], adot3);
        } else {
          irr2[d] = dadd(irr2[d], adot2);
          irr3[d] = dadd(irr3[d], adot3);
        }
      }
    }
  }
  if (!valid) return;
  double *o = out + 12 * (size_t)i;
  for (int d = 0; d < 3; ++d) {
    o[d] = reg2[d];
    o[3 + d] = reg3[d];
    o[6 + d] = irr2[d];
    o[9 + d] = irr3[d];
  }
}

}  // namespace

void launch_init_derivs23(cudaStream_t s, int n, const double *x, const double *v, const double *a0,
                          const double *a1, const double *mass, const double *r2nb, double eps2,
                          double *out) {
  const int blocks = (n + kInitThreads - 1) / kInitThreads;
  init_derivs23_kernel<<<blocks, kInitThreads, 0, s>>>(n, x, v, a0, a1, mass, r2nb, eps2, out);
}

}  // namespace abyss
