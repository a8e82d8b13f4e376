// Per-neighbour terms of the irregular force (ComputeAcceleration.cpp:14-190 as
// restated in ac_integrator.cpp): prediction of each neighbour to the common new
// time, then m r^-3 x and m r^-3 (v - 3 (x.v) x / r^2) with softened r^2, each
// neighbour independent of the others.  The caller adds the terms in neighbour
// order, so the sums are the same, bit for bit, as the one-pass loop.
//
// Plain C++ compiled by g++ with -ffp-contract=off (no fused multiply-add, the
// operations exactly as written); target_clones builds AVX-512, AVX2 and
// baseline versions and picks one for the host's CPU at load time.
#include <cmath>

namespace abyss_host {

__attribute__((target_clones("avx512f", "avx2", "default")))
void irregular_terms(int nn, const double *X, const double *V, const double *A0, const double *A1, const double *T,
                     const double *M, const double *pos, const double *vel, double new_time, double scale,
                     double eps2, double *ta, double *tj) {
  for (int k = 0; k < nn; ++k) {
    const double dt = (new_time - T[k]) * scale;
    double x[3], v[3], r2 = 0.0, vx = 0.0;
    for (int d = 0; d < 3; ++d) {
      double pj, vj;
      if (dt == 0) {
        pj = X[3 * k + d];
        vj = V[3 * k + d];
      } else {
        pj = ((A1[3 * k + d] * dt / 3 + A0[3 * k + d]) * dt / 2 + V[3 * k + d]) * dt + X[3 * k + d];
        vj = (A1[3 * k + d] * dt / 2 + A0[3 * k + d]) * dt + V[3 * k + d];
      }
      x[d] = pj - pos[d];
      v[d] = vj - vel[d];
      r2 += x[d] * x[d];
      vx += v[d] * x[d];
    }
    const double r2s = r2 + eps2;
    const double m_r3 = M[k] / (r2s * std::sqrt(r2s));
    for (int d = 0; d < 3; ++d) {
      ta[3 * k + d] = m_r3 * x[d];
      tj[3 * k + d] = m_r3 * (v[d] - 3 * x[d] * vx / r2s);
    }
  }
}

}  // namespace abyss_host
