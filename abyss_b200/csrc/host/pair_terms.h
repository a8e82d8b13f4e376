// Per-neighbour terms of the host's irregular step (host/pair_terms.cpp).
#pragma once

namespace abyss_host {

// A neighbour's fields as its irregular step reads them, on two cache lines:
// position, velocity, mass, the time it was last advanced to, and the first
// two derivatives of its total acceleration.
struct alignas(64) NbRec {
  double x[3], v[3], m, t;
  double a0[3], a1[3], pad[2];
};

// For the nn neighbours nb[k] (records rec[slot[nb[k]]]) of a particle at
// pos/vel: each neighbour predicted to new_time, then m r^-3 x into ta[3k..]
// and m r^-3 (v - 3 (x.v) x / r^2) into tj[3k..], r^2 softened by eps2.
void irregular_terms(int nn, const int *nb, const int *slot, const NbRec *rec, const double *pos, const double *vel,
                     double new_time, double scale, double eps2, double *ta, double *tj);

}  // namespace abyss_host
