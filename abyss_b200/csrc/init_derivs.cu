// Second and third time derivatives of the acceleration at a common time, the
// initialisation pass of the Ahmad-Cohen scheme (CalculateAcceleration23,
// src_mpi/Particle/Initialize.cpp:102-185), split into a regular part
// (r^2 >= R^2, unsoftened) and an irregular part, with eps2 added to r^2 in the
// force terms.
//
// One warp owns one target.  Its 32 lanes compute the terms of 32 consecutive
// j at once, every operation in the reference's order and rounded to nearest
// (__dadd_rn etc.; this file is also compiled with -fmad=false); lanes 0-5 then
// add the chunk's terms into the six sums (2 derivatives x 3 dimensions; a
// regular and an irregular sum each) in ascending j.  Each sum therefore sees
// the same terms in the same order as the sequential FP64 host loop and equals
// it bit for bit, while the O(N^2) term work (about 25 FP64 divisions per pair)
// is spread over every lane of the GPU.
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace abyss {

namespace {

constexpr int kInitWarps = 4;  // targets per block
constexpr int kInitThreads = 32 * kInitWarps;

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
  // per warp: the chunk's terms [component][lane] and each lane's kind
  // (0: no term, 1: regular, 2: irregular)
  __shared__ double s_term[kInitWarps][6][32];
  __shared__ int s_kind[kInitWarps][32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kInitWarps + w;
  if (i >= n) return;  // the whole warp: no block-wide barrier below
  double xi[3], vi[3], a1i[3], a1doti[3];
  for (int d = 0; d < 3; ++d) {
    xi[d] = x[3 * i + d];
    vi[d] = v[3 * i + d];
    a1i[d] = a0[3 * i + d];
    a1doti[d] = a1[3 * i + d];
  }
  const double R2 = r2nb[i];
  // lane c < 6 owns component c: derivative c / 3 (2nd, 3rd), dimension c % 3
  double sum_reg = 0.0, sum_irr = 0.0;

  for (int j0 = 0; j0 < n; j0 += 32) {
    const int j = j0 + lane;
    int kind = 0;
    double t2[3] = {0, 0, 0}, t3[3] = {0, 0, 0};
    if (j < n && j != i) {
      double xx[3], vv[3], a21[3], a21dot[3];
      double r2u = 0.0, vr = 0.0, v2 = 0.0, rdf_r2 = 0.0, vdf_r2 = 0.0, rdfdot_r2 = 0.0;
      for (int d = 0; d < 3; ++d) {
        xx[d] = dsub(x[3 * j + d], xi[d]);
        vv[d] = dsub(v[3 * j + d], vi[d]);
        r2u = dadd(r2u, dmul(xx[d], xx[d]));
        vr = dadd(vr, dmul(vv[d], xx[d]));
        v2 = dadd(v2, dmul(vv[d], vv[d]));
      }
      const double r2 = dadd(r2u, eps2);
      const double r3 = dmul(r2, __dsqrt_rn(r2));
      const double mj = mass[j];
      const double m_r3 = ddiv(mj, r3);
      double da[3], dd[3];
      for (int d = 0; d < 3; ++d) {
        da[d] = dsub(a1i[d], a0[3 * j + d]);
        dd[d] = dsub(a1doti[d], a1[3 * j + d]);
        a21[d] = dmul(m_r3, xx[d]);
        // m_r3 * (v - 3 * x * vr / r2)
        a21dot[d] = dmul(m_r3, dsub(vv[d], ddiv(dmul(dmul(3.0, xx[d]), vr), r2)));
        rdf_r2 = dadd(rdf_r2, ddiv(dmul(xx[d], da[d]), r2));
        vdf_r2 = dadd(vdf_r2, ddiv(dmul(vv[d], da[d]), r2));
        rdfdot_r2 = dadd(rdfdot_r2, ddiv(dmul(xx[d], dd[d]), r2));
      }
      const double a = ddiv(vr, r2);
      // b = v2 / r2 + rdf_r2 + a * a
      const double b = dadd(dadd(ddiv(v2, r2), rdf_r2), dmul(a, a));
      // c = 3 * vdf_r2 + rdfdot_r2 + a * (3 * b - 4 * a * a)
      const double c = dadd(dadd(dmul(3.0, vdf_r2), rdfdot_r2), dmul(a, dsub(dmul(3.0, b), dmul(dmul(4.0, a), a))));
      for (int d = 0; d < 3; ++d) {
        // adot2 = -m * da / r3 - 6 * a * a21dot - 3 * b * a21
        t2[d] = dsub(dsub(ddiv(dmul(-mj, da[d]), r3), dmul(dmul(6.0, a), a21dot[d])), dmul(dmul(3.0, b), a21[d]));
        // adot3 = -m * dd / r3 - 9 * a * adot2 - 9 * b * a21dot - 3 * c * a21
        t3[d] = dsub(dsub(dsub(ddiv(dmul(-mj, dd[d]), r3), dmul(dmul(9.0, a), t2[d])), dmul(dmul(9.0, b), a21dot[d])),
                     dmul(dmul(3.0, c), a21[d]));
      }
      kind = r2u < R2 ? 2 : 1;
    }
    for (int d = 0; d < 3; ++d) {
      s_term[w][d][lane] = t2[d];
      s_term[w][3 + d][lane] = t3[d];
    }
    s_kind[w][lane] = kind;
    __syncwarp();
    if (lane < 6) {
      const int cnt = min(32, n - j0);
      for (int k = 0; k < cnt; ++k) {
        const int f = s_kind[w][k];
        const double val = s_term[w][lane][k];
        if (f == 1)
          sum_reg = dadd(sum_reg, val);
        else if (f == 2)
          sum_irr = dadd(sum_irr, val);
      }
    }
    __syncwarp();
  }
  if (lane < 6) {
    // out row: reg2[3], reg3[3], irr2[3], irr3[3]
    double *o = out + 12 * (size_t)i;
    o[lane] = sum_reg;
    o[6 + lane] = sum_irr;
  }
}

}  // namespace

void launch_init_derivs23(cudaStream_t s, int n, const double *x, const double *v, const double *a0,
                          const double *a1, const double *mass, const double *r2nb, double eps2,
                          double *out) {
  const int blocks = (n + kInitWarps - 1) / kInitWarps;
  init_derivs23_kernel<<<blocks, kInitThreads, 0, s>>>(n, x, v, a0, a1, mass, r2nb, eps2, out);
}

}  // namespace abyss
