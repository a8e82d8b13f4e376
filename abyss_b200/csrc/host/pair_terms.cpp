// Per-neighbour terms of the irregular force (ComputeAcceleration.cpp:14-190 as
// restated in ac_integrator.cpp): prediction of each neighbour to the common new
// time, then m r^-3 x and m r^-3 (v - 3 (x.v) x / r^2) with softened r^2, each
// neighbour independent of the others.  The caller adds the terms in neighbour
// order, so the sums are the same, bit for bit, as the one-pass loop.
//
// Plain C++ compiled by g++ with -ffp-contract=off (no fused multiply-add, the
// operations exactly as written) and -fno-math-errno (sqrt as the correctly
// rounded instruction, without the errno call that blocks vectorisation);
// target_clones builds AVX-512, AVX2 and baseline versions and picks one for
// the host's CPU at load time.  The loop body has no branch: the predicted
// state is computed for every neighbour and selected, so the compiler
// vectorises across neighbours, gathering each neighbour's record itself.
#include <cmath>

#include "pair_terms.h"

namespace abyss_host {

__attribute__((target_clones("avx512f", "avx2", "default")))
void irregular_terms(int nn, const int *__restrict nb, const int *__restrict slot, const NbRec *__restrict rec,
                     const double *__restrict pos, const double *__restrict vel, double new_time, double scale,
                     double eps2, double *__restrict ta, double *__restrict tj) {
  const double pi[3] = {pos[0], pos[1], pos[2]}, vi[3] = {vel[0], vel[1], vel[2]};
  for (int k = 0; k < nn; ++k) {
    const NbRec &q = rec[slot[nb[k]]];
    const double dt = (new_time - q.t) * scale;
    double x[3], v[3], r2 = 0.0, vx = 0.0;
    for (int d = 0; d < 3; ++d) {
      // a neighbour already at new_time keeps its state exactly
      const double pp = ((q.a1[d] * dt / 3 + q.a0[d]) * dt / 2 + q.v[d]) * dt + q.x[d];
      const double vp = (q.a1[d] * dt / 2 + q.a0[d]) * dt + q.v[d];
      const double pj = dt == 0 ? q.x[d] : pp;
      const double vj = dt == 0 ? q.v[d] : vp;
      x[d] = pj - pi[d];
      v[d] = vj - vi[d];
      r2 += x[d] * x[d];
      vx += v[d] * x[d];
    }
    const double r2s = r2 + eps2;
    const double m_r3 = q.m / (r2s * std::sqrt(r2s));
    for (int d = 0; d < 3; ++d) {
      ta[3 * k + d] = m_r3 * x[d];
      tj[3 * k + d] = m_r3 * (v[d] - 3 * x[d] * vx / r2s);
    }
  }
}

}  // namespace abyss_host
