// Irregular steps on the device (irregular.h): the level loop of the
// Ahmad-Cohen irregular force in one persistent cooperative kernel; and the
// rest of a block -- the next block's particles, the regular corrector, commit,
// time steps and radii -- for integrations whose state stays on the device
// (the blk_* kernels below).
//
// The host integrator runs, between two regular blocks, every particle whose
// next irregular time is due, level by level in increasing block time
// (src_mpi/RootRoutines.cpp:488-1005 as restated in host/ac_integrator.cpp
// irregular_levels).  Here that loop runs on the GPU, one level per iteration:
//
//   B  every particle of the level is stepped from the pre-level state, one
//      warp per particle: its prediction, its neighbours' prediction to the
//      common new time and their FP64 pair terms (lanes over neighbours), the
//      terms added in neighbour order, the Hermite corrector and the new
//      irregular level (ComputeAcceleration.cpp:14-190,
//      UpdateParticle.cpp:151-241); results go to a per-particle pending slot;
//   -- grid barrier --
//   C  the level is committed (IrrUpdate, WorkerRoutines.cpp:76-87) and the
//      next level is found: the minimum next block time still due;
//   -- grid barrier --
//
// Every expression keeps the host integrator's operation order and the file is
// compiled without multiply-add contraction, so a step equals the host's bit
// for bit: IEEE add, multiply, divide and square root are exact-rounded on both
// sides.  The one library function is log, in the level rule
// floor(log(dt / scale) / log(2)); the divisor log(2) is the host's value, and
// level decisions whose quotient lies within 1e-12 of an integer -- the only
// ones where a last-place difference between the device's and the host's log
// could change the level -- are counted and reported.
//
// The grid barrier is one arrive counter whose top bit flips when the last
// block arrives; its waits are bounded (about a second), after which the kernel
// records ABYSS_ERR_TIMEOUT and every block leaves.  Values written in the loop are read back with
// L2-coherent loads (__ldcg): an SM's L1 does not see other SMs' stores.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/abyss_reg.h"
#include "irregular.h"

namespace abyss_irr {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxSlice = 4096;  // particles per block of the level loop
constexpr int kBad = 1;       // a time step out of range
constexpr int kTimeout = 2;   // a grid-barrier wait ran out
constexpr int kBadIndex = 4;  // an uploaded image named a particle outside the cluster
constexpr int kRegBad = 8;    // a regular block's time step out of range
constexpr int kSchedChunk = 2048;  // particles per block of the block-scheduling kernels (256 x 8)
constexpr long long kBarrierSpins = 5000000;  // x up to 256 ns sleep: about a second

// A particle as its neighbours' steps read it (one 128-byte line).
struct __align__(128) Rec {
  double x[3], v[3], m, t;
  double a0[3], a1[3];  // a_tot[.][0], a_tot[.][1]
  double pad[2];
};

struct Pend {
  double nx[3], nv[3];
  double a_irr[12], a_tot[12];
  double dt_irr;
  ULL tb_irr, new_cur;
  int lv_irr, move;
};

// A regular block's corrector results for one target, committed once every
// target's corrector has run (the host integrator's Pending).
struct RPend {
  double nx[3], nv[3];
  double a_reg[12], a_irr[12], a_tot[12];
};

struct Ctl {
  ULL tmin;  // the next regular block's time (engine_next_block)
  int m, pad2;  // and its number of particles
  ULL lmin[2];
  unsigned bar_count, bar_unused;
  int status, pad;
  long long levels, steps, borderline;
  int mcount[2];  // members of the level (alternating slots)
  // SM clock cycles of block 0 in each part of a level, summed over levels:
  // [0] member list, [1] (unused), [2] steps, [3] their barrier,
  // [4] commit and next level, [5] its barrier
  long long cycles[6];
};

struct State {
  int n, cap;
  Rec *rec;
  double *a_tot, *a_reg, *a_irr, *t_reg, *dt_irr;
  ULL *cur_irr, *tb_irr, *next_irr, *new_cur_irr, *cur_reg, *tb_reg;
  int *lv_irr, *lv_reg, *nnb, *nb, *touched;
  int *members;   // the level's particles, in any order
  double *r2nb, *dt_reg;  // read and written by whole regular blocks only
  int *tg;        // the regular block's particles, ascending
  int *bcnt;      // per scheduling block: its particles due
  RPend *rpend;   // [m] regular corrector results
  Pend *pend;
  Ctl *ctl;
  Image *img;     // device staging of images
  int *lists;     // device staging of lists, packed
  Changed *chg;   // device staging of changed fields [n]
};

// ------------------------------------------------------------ the step itself

__device__ __forceinline__ double pow2d(int e) { return ldexp(1.0, e); }
__device__ __forceinline__ ULL pow2_blocks(int e) { return (ULL)ldexp(1.0, e); }

__device__ __forceinline__ void load_rec(const Rec *r, double (&x)[3], double (&v)[3], double &m, double &t,
                                         double (&a0)[3], double (&a1)[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    x[d] = __ldcg(&r->x[d]);
    v[d] = __ldcg(&r->v[d]);
    a0[d] = __ldcg(&r->a0[d]);
    a1[d] = __ldcg(&r->a1[d]);
  }
  m = __ldcg(&r->m);
  t = __ldcg(&r->t);
}

// TimeStepRoutines.cpp:28-63 (host/ac_integrator.cpp new_step_irr).
__device__ double new_step_irr(const double *f, const double *df, double eta) {
  const double F2 = f[0] * f[0] + f[4] * f[4] + f[8] * f[8];
  const double Fdot2 = df[1] * df[1] + df[5] * df[5] + df[9] * df[9];
  const double F2dot2 = df[2] * df[2] + df[6] * df[6] + df[10] * df[10];
  const double F3dot2 = df[3] * df[3] + df[7] * df[7] + df[11] * df[11];
  const double ts = (sqrt(F2 * F2dot2) + Fdot2) / (sqrt(Fdot2 * F3dot2) + F2dot2);
  return sqrt(eta * ts);
}

// TimeStepRoutines.cpp:102-115 (block_step): the level only.
__device__ int block_level(const Params &P, double dt, long long &border) {
  const double q = log(dt / P.scale) / P.ln2;
  if (fabs(q - rint(q)) < 1e-12 * fmax(1.0, fabs(q))) ++border;
  int level = (int)floor(q);
  if (level < P.time_block) level = P.time_block;
  return level;
}

// UpdateParticle.cpp:151-241 (host/ac_integrator.cpp time_step_irr_of); lv,
// dt, tb are updated in place.  Returns false for a step out of range.
__device__ bool level_irr(const Params &P, bool has_nb, const double *a_tot, const double *a_irr, ULL new_cur,
                          ULL cur_reg, ULL tb_reg, int lv_reg, int &lv_irr, double &dt_irr, ULL &tb_irr,
                          long long &border) {
  if (!has_nb) {
    lv_irr = lv_reg;
    dt_irr = pow2d(lv_reg);
    tb_irr = pow2_blocks(lv_reg - P.time_block);
    return true;
  }
  int lv = block_level(P, new_step_irr(a_tot, a_irr, P.eta_irr), border);
  ULL tb = pow2_blocks(lv - P.time_block);
  const int p_lv = lv_irr;
  const ULL p_tb = tb_irr;
  if (lv > p_lv) {
    if (fmod((double)new_cur, 2.0 * (double)p_tb) == 0) {
      lv = p_lv + 1;
      tb = 2 * p_tb;
    } else {
      lv = p_lv;
      tb = p_tb;
    }
  } else if (lv < p_lv) {
    if (lv < p_lv - 1) {
      lv = p_lv - 2;
      tb = p_tb / 4;
    } else {
      lv = p_lv - 1;
      tb = p_tb / 2;
    }
  } else {
    lv = p_lv;
    tb = p_tb;
  }
  const ULL reg_end = cur_reg + tb_reg;
  // ends within (lv - lv_reg + 1) + 64 rounds: lv falls by one and tb halves
  for (int guard = 0; ((new_cur < reg_end) && (new_cur + tb > reg_end)) || (lv >= lv_reg); ++guard) {
    if (guard > 4096) return false;
    lv--;
    tb = (ULL)(tb * 0.5);
  }
  lv_irr = max(P.time_block, lv);
  dt_irr = pow2d(lv_irr);
  tb_irr = pow2_blocks(lv_irr - P.time_block);
  return !(dt_irr > 1);
}

// One neighbour's terms (host/pair_terms.cpp irregular_terms): j predicted to
// new_time, then m r^-3 x and m r^-3 (v - 3 (x.v) x / r^2), r^2 softened.
__device__ __forceinline__ void pair_terms(const Rec *q, double new_time, double scale, double eps2,
                                           const double (&pi)[3], const double (&vi)[3], double (&ta)[3],
                                           double (&tj)[3]) {
  double qx[3], qv[3], qm, qt, qa0[3], qa1[3];
  load_rec(q, qx, qv, qm, qt, qa0, qa1);
  const double dt = (new_time - qt) * scale;
  double x[3], v[3], r2 = 0.0, vx = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double pp = ((qa1[d] * dt / 3 + qa0[d]) * dt / 2 + qv[d]) * dt + qx[d];
    const double vp = (qa1[d] * dt / 2 + qa0[d]) * dt + qv[d];
    const double pj = dt == 0 ? qx[d] : pp;
    const double vj = dt == 0 ? qv[d] : vp;
    x[d] = pj - pi[d];
    v[d] = vj - vi[d];
    r2 += x[d] * x[d];
    vx += v[d] * x[d];
  }
  const double r2s = r2 + eps2;
  const double m_r3 = qm / (r2s * sqrt(r2s));
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    ta[d] = m_r3 * x[d];
    tj[d] = m_r3 * (v[d] - 3 * x[d] * vx / r2s);
  }
}

// Particle i's irregular step from the state as it stands, by one warp (every
// lane ends with the same results; lane 0's copy is the one stored); `terms` is
// the warp's shared scratch of 6 x 64 doubles.  Returns false for a time step
// out of range.
__device__ bool member_step(const State &S, const Params &P, int i, Pend &pd, long long &border, double *terms) {
  const int lane = threadIdx.x & 31;
  // every load the step needs is issued first: they are independent, and the
  // step is a chain of L2 round trips otherwise
  const int nn = S.nnb[i];
  const int *nb = S.nb + (size_t)i * S.cap;
  int j0 = lane < nn ? nb[lane] : -1;
  int j1 = 32 + lane < nn ? nb[32 + lane] : -1;
  double at[12], ai[12], ar[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    at[k] = __ldcg(&S.a_tot[12 * (size_t)i + k]);
    ai[k] = __ldcg(&S.a_irr[12 * (size_t)i + k]);
    ar[k] = S.a_reg[12 * (size_t)i + k];
  }
  const double dt_irr = __ldcg(&S.dt_irr[i]);
  const double t_reg = S.t_reg[i];
  const int lv0 = __ldcg(&S.lv_irr[i]);
  const ULL tb0 = __ldcg(&S.tb_irr[i]), cur0 = __ldcg(&S.cur_irr[i]);
  const ULL cur_reg = S.cur_reg[i], tb_reg = S.tb_reg[i];
  const int lv_reg = S.lv_reg[i];
  double x[3], v[3], m, t, a0[3], a1[3];
  load_rec(&S.rec[i], x, v, m, t, a0, a1);
  if (nn == 0) {
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      pd.a_tot[k] = at[k];
      pd.a_irr[k] = ai[k];
    }
    pd.move = 0;
  } else {
    pd.move = 1;
    const double new_time = t + dt_irr;
    const double dt = dt_irr * P.scale;
    double pos[3], vel[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (dt == 0) {
        pos[d] = x[d];
        vel[d] = v[d];
      } else {
        pos[d] = ((at[4 * d + 1] * dt / 3 + at[4 * d + 0]) * dt / 2 + v[d]) * dt + x[d];
        vel[d] = (at[4 * d + 1] * dt / 2 + at[4 * d + 0]) * dt + v[d];
      }
    }
    // 64 neighbours a round, two per lane; lane c < 6 then adds component c of
    // the round's terms in neighbour order: exactly the host's sequential sums
    double sum = 0.0;
    for (int base = 0; base < nn; base += 64) {
      if (base > 0) {
        j0 = base + lane < nn ? nb[base + lane] : -1;
        j1 = base + 32 + lane < nn ? nb[base + 32 + lane] : -1;
      }
      double ta[3] = {0.0, 0.0, 0.0}, tj[3] = {0.0, 0.0, 0.0};
      double ua[3] = {0.0, 0.0, 0.0}, uj[3] = {0.0, 0.0, 0.0};
      if (j0 >= 0) pair_terms(&S.rec[j0], new_time, P.scale, P.eps2, pos, vel, ta, tj);
      if (j1 >= 0) pair_terms(&S.rec[j1], new_time, P.scale, P.eps2, pos, vel, ua, uj);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        terms[d * 64 + lane] = ta[d];
        terms[(3 + d) * 64 + lane] = tj[d];
        terms[d * 64 + 32 + lane] = ua[d];
        terms[(3 + d) * 64 + 32 + lane] = uj[d];
      }
      __syncwarp();
      const int cnt = min(64, nn - base);
      if (lane < 6)
        for (int l = 0; l < cnt; ++l) sum += terms[lane * 64 + l];
      __syncwarp();
    }
    double a_tmp[3], adot_tmp[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      a_tmp[d] = __shfl_sync(0xffffffffu, sum, d);
      adot_tmp[d] = __shfl_sync(0xffffffffu, sum, 3 + d);
    }
    const double dt_ex = (new_time - t_reg) * P.scale;
    const double dt2 = dt * dt, dt3 = dt2 * dt, dt4 = dt3 * dt, dt5 = dt4 * dt;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double da_dt2 = (ai[4 * d + 0] - a_tmp[d]) / dt2;
      const double adot_dt = (ai[4 * d + 1] + adot_tmp[d]) / dt;
      const double a2 = -6 * da_dt2 - 2 * adot_dt - 2 * ai[4 * d + 1] / dt;
      const double a3 = (12 * da_dt2 + 6 * adot_dt) / dt;
      pd.nx[d] = pos[d] + a2 * dt4 / 24 + a3 * dt5 / 120;
      pd.nv[d] = vel[d] + a2 * dt3 / 6 + a3 * dt4 / 24;
      pd.a_irr[4 * d + 0] = a_tmp[d];
      pd.a_irr[4 * d + 1] = adot_tmp[d];
      pd.a_irr[4 * d + 2] = a2;
      pd.a_irr[4 * d + 3] = a3;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      pd.a_tot[4 * d + 0] = ar[4 * d + 0] + pd.a_irr[4 * d + 0] + ar[4 * d + 1] * dt_ex;
      pd.a_tot[4 * d + 1] = ar[4 * d + 1] + pd.a_irr[4 * d + 1];
      pd.a_tot[4 * d + 2] = ar[4 * d + 2] + pd.a_irr[4 * d + 2];
      pd.a_tot[4 * d + 3] = ar[4 * d + 3] + pd.a_irr[4 * d + 3];
    }
  }
  // the new level from the new derivatives (WorkerRoutines.cpp:46-64)
  pd.lv_irr = lv0;
  pd.dt_irr = dt_irr;
  pd.tb_irr = tb0;
  pd.new_cur = cur0 + tb0;
  return level_irr(P, nn > 0, pd.a_tot, pd.a_irr, pd.new_cur, cur_reg, tb_reg, lv_reg, pd.lv_irr, pd.dt_irr,
                   pd.tb_irr, border);
}

__device__ void store_pend(Pend *dst, const Pend &pd) {
  for (int d = 0; d < 3; ++d) {
    dst->nx[d] = pd.nx[d];
    dst->nv[d] = pd.nv[d];
  }
  for (int k = 0; k < 12; ++k) {
    dst->a_irr[k] = pd.a_irr[k];
    dst->a_tot[k] = pd.a_tot[k];
  }
  dst->dt_irr = pd.dt_irr;
  dst->tb_irr = pd.tb_irr;
  dst->new_cur = pd.new_cur;
  dst->lv_irr = pd.lv_irr;
  dst->move = pd.move;
}

// IrrUpdate: commit particle i's pending step; returns its next block time.
// Every pending field is loaded before the first store: with loads and stores
// interleaved the compiler cannot tell them apart (possible aliasing) and would
// run some thirty L2 round trips one after another.
__device__ ULL commit(const State &S, const Params &P, int i) {
  const Pend *q = &S.pend[i];
  const int lv = __ldcg(&q->lv_irr);
  const int move = __ldcg(&q->move);
  const double dtv = __ldcg(&q->dt_irr);
  const ULL tb = __ldcg(&q->tb_irr), nc = __ldcg(&q->new_cur);
  double at[12], ai[12], nx[3], nv[3];
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    at[k] = __ldcg(&q->a_tot[k]);
    ai[k] = __ldcg(&q->a_irr[k]);
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    nx[d] = __ldcg(&q->nx[d]);
    nv[d] = __ldcg(&q->nv[d]);
  }
  const int nn = S.nnb[i];
  S.lv_irr[i] = lv;
  S.dt_irr[i] = dtv;
  S.tb_irr[i] = tb;
  S.new_cur_irr[i] = nc;
  Rec *r = &S.rec[i];
#pragma unroll
  for (int k = 0; k < 12; ++k) {
    S.a_tot[12 * (size_t)i + k] = at[k];
    S.a_irr[12 * (size_t)i + k] = ai[k];
  }
  const ULL next = nc + tb;
  S.next_irr[i] = next;
  if (nn > 0 && move) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      r->x[d] = nx[d];
      r->v[d] = nv[d];
    }
  }
  S.cur_irr[i] = nc;
  r->t = (double)nc * P.time_step;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    r->a0[d] = at[4 * d + 0];
    r->a1[d] = at[4 * d + 1];
  }
  S.touched[i] = 1;
  return next;
}

// ------------------------------------------------------------ grid barrier

__device__ __forceinline__ int ld_volatile(const int *p) { return *(volatile const int *)p; }

// Every block of the (co-resident) grid arrives; returns false when this
// block's wait ran out (the others' waits then run out too, and every block
// leaves the loop).
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned *p, unsigned a) {
  unsigned old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(a) : "memory");
  return old;
}

// One atomic per block: block 0 adds 2^31 - (blocks - 1), every other block 1,
// so that the counter's top bit flips exactly when the last block has arrived
// (its low bits return to where they were).  A block waits for the flip of the
// bit its own atomic saw.
__device__ bool grid_barrier(Ctl *ctl) {
  __shared__ int s_ok;
  // the block's writes are ordered before thread 0's release by the block
  // barrier; its acquire orders every later read of the block after the other
  // blocks' releases (release/acquire at GPU scope are cumulative)
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned inc = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1) : 1u;
    const unsigned old = atom_add_acq_rel(&ctl->bar_count, inc);
    long long spins = 0;
    unsigned nap = 0;
    while (((ld_acquire(&ctl->bar_count) ^ old) & 0x80000000u) == 0) {
      if (++spins > kBarrierSpins) {
        atomicOr(&ctl->status, kTimeout);
        ok = 0;
        break;
      }
      // a level's barrier is usually a few microseconds: poll, then back off
      if (spins > 64) {
        nap = nap < 256 ? nap + 32 : 256;
        __nanosleep(nap);
      }
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ ULL block_min(ULL v) {
  __shared__ ULL s_min[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) s_min[w] = v;
  __syncthreads();
  ULL r = ULLONG_MAX;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = min(r, s_min[k]);
  __syncthreads();
  return r;
}

// ------------------------------------------------------------ kernels

// The level loop up to P.next_reg_block (cooperative launch: every block
// resident).  Block b owns the particles [b * slice, (b + 1) * slice): it finds
// the level's members among them, steps them with its own warps and commits
// them, so that a level needs two grid barriers -- after the steps (no commit
// may change a neighbour another block still reads) and after the commits (the
// next level is the minimum over every block's particles).
__global__ void __launch_bounds__(kThreads) irr_levels(State S, Params P, int slice) {
  __shared__ double s_terms[kThreads / 32][6 * 64];
  __shared__ int s_mem[kMaxSlice];
  __shared__ int s_cnt;
  Ctl *ctl = S.ctl;
  const int tid = threadIdx.x, lane = tid & 31, wib = tid >> 5, nwb = blockDim.x >> 5;
  const int b0 = blockIdx.x * slice, b1 = min(S.n, b0 + slice);
  double *terms = s_terms[wib];
  const bool clerk = blockIdx.x == 0 && tid == 0;  // keeps the counters
  long long cyc[6] = {0, 0, 0, 0, 0, 0};
  // the first level: the smallest next block time still due
  ULL mn = ULLONG_MAX;
  for (int i = b0 + tid; i < b1; i += blockDim.x) {
    const ULL t = __ldcg(&S.next_irr[i]);
    if (t <= P.next_reg_block && t < mn) mn = t;
  }
  mn = block_min(mn);
  if (tid == 0 && mn != ULLONG_MAX) atomicMin(&ctl->lmin[0], mn);
  if (!grid_barrier(ctl)) return;
  int parity = 0;
  long long border = 0;
  for (;;) {
    const ULL lvl = *(volatile ULL *)&ctl->lmin[parity];
    if (lvl == ULLONG_MAX) break;
    const long long t0 = clock64();
    // the slot of the next level's minimum was last read before the previous
    // barrier: clear it
    if (clerk) {
      ctl->lmin[parity ^ 1] = ULLONG_MAX;
      ctl->levels++;
    }
    // this block's members of the level (any order: each is stepped from the
    // pre-level state alone)
    if (tid == 0) s_cnt = 0;
    __syncthreads();
    for (int i = b0 + tid; i < b1; i += blockDim.x)
      if (__ldcg(&S.next_irr[i]) == lvl) s_mem[atomicAdd(&s_cnt, 1)] = i;
    __syncthreads();
    const int cnt = s_cnt;
    const long long t1 = clock64();
    // B: the members, one warp each
    for (int k = wib; k < cnt; k += nwb) {
      const int i = s_mem[k];
      Pend pd{};
      const bool ok = member_step(S, P, i, pd, border, terms);
      if (lane == 0) {
        store_pend(&S.pend[i], pd);
        if (!ok) atomicOr(&ctl->status, kBad);
      }
    }
    const long long t2 = clock64();
    if (!grid_barrier(ctl)) break;
    const long long t3 = clock64();
    // a step out of range: nothing of this level is committed.  The status
    // word is only set in B, so every block reads the same value here.
    if (ld_volatile(&ctl->status) & kBad) break;
    // C: commit this block's members, and the next level's block time
    ULL nx = ULLONG_MAX;
    for (int i = b0 + tid; i < b1; i += blockDim.x) {
      ULL t = __ldcg(&S.next_irr[i]);
      if (t == lvl) t = commit(S, P, i);
      if (t <= P.next_reg_block && t < nx) nx = t;
    }
    nx = block_min(nx);
    if (tid == 0) {
      if (nx != ULLONG_MAX) atomicMin(&ctl->lmin[parity ^ 1], nx);
      if (cnt) atomicAdd((unsigned long long *)&ctl->steps, (unsigned long long)cnt);
    }
    parity ^= 1;
    const long long t4 = clock64();
    if (!grid_barrier(ctl)) break;
    const long long t5 = clock64();
    cyc[0] += t1 - t0;
    cyc[2] += t2 - t1;
    cyc[3] += t3 - t2;
    cyc[4] += t4 - t3;
    cyc[5] += t5 - t4;
  }
  if (clerk)
    for (int q = 0; q < 6; ++q) ctl->cycles[q] += cyc[q];
  // every lane of a warp stepped the same particles: lane 0's count is the warp's
  if (lane == 0 && border) atomicAdd((unsigned long long *)&ctl->borderline, (unsigned long long)border);
}

// Single steps of listed particles (nothing committed), one warp each.
__global__ void __launch_bounds__(kThreads) irr_steps(State S, Params P, int count, const int *idx, double *out_pos,
                                                     double *out_vel, double *out_airr, double *out_atot,
                                                     int *out_lv, double *out_dt, ULL *out_tb) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  __shared__ double s_terms[kThreads / 32][6 * 64];
  double *terms = s_terms[threadIdx.x >> 5];
  long long border = 0;
  for (int k = warp; k < count; k += nwarps) {
    const int i = idx[k];
    Pend pd{};
    const bool ok = member_step(S, P, i, pd, border, terms);
    if (lane == 0) {
      for (int d = 0; d < 3; ++d) {
        out_pos[3 * (size_t)k + d] = pd.move ? pd.nx[d] : S.rec[i].x[d];
        out_vel[3 * (size_t)k + d] = pd.move ? pd.nv[d] : S.rec[i].v[d];
      }
      for (int q = 0; q < 12; ++q) {
        out_airr[12 * (size_t)k + q] = pd.a_irr[q];
        out_atot[12 * (size_t)k + q] = pd.a_tot[q];
      }
      out_lv[k] = pd.lv_irr;
      out_dt[k] = pd.dt_irr;
      out_tb[k] = pd.tb_irr;
      if (!ok) atomicOr(&S.ctl->status, kBad);
    }
  }
  if (lane == 0 && border) atomicAdd((unsigned long long *)&S.ctl->borderline, (unsigned long long)border);
}

// Scatter staged images (and their lists) into the state.
__global__ void irr_scatter(State S, int count) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const Image &g = S.img[k];
    const int i = g.index;
    if (i < 0 || i >= S.n || g.nnb < 0 || g.nnb > S.cap) {
      atomicOr(&S.ctl->status, kBadIndex);
      continue;
    }
    Rec &r = S.rec[i];
    for (int d = 0; d < 3; ++d) {
      r.x[d] = g.x[d];
      r.v[d] = g.v[d];
      r.a0[d] = g.a_tot[4 * d + 0];
      r.a1[d] = g.a_tot[4 * d + 1];
    }
    r.m = g.m;
    r.t = g.t_irr;
    for (int q = 0; q < 12; ++q) {
      S.a_tot[12 * (size_t)i + q] = g.a_tot[q];
      S.a_reg[12 * (size_t)i + q] = g.a_reg[q];
      S.a_irr[12 * (size_t)i + q] = g.a_irr[q];
    }
    S.t_reg[i] = g.t_reg;
    S.dt_irr[i] = g.dt_irr;
    S.r2nb[i] = g.r2nb;
    S.dt_reg[i] = g.dt_reg;
    S.cur_irr[i] = g.cur_irr;
    S.tb_irr[i] = g.tb_irr;
    S.next_irr[i] = g.next_irr;
    S.new_cur_irr[i] = g.new_cur_irr;
    S.cur_reg[i] = g.cur_reg;
    S.tb_reg[i] = g.tb_reg;
    S.lv_irr[i] = g.lv_irr;
    S.lv_reg[i] = g.lv_reg;
    int bad = 0;
    for (int q = 0; q < g.nnb; ++q) {
      const int j = S.lists[g.list_off + q];
      bad |= (j < 0 || j >= S.n);
      S.nb[(size_t)i * S.cap + q] = j;
    }
    // a neighbour outside the cluster is refused, and never read
    S.nnb[i] = bad ? 0 : g.nnb;
    if (bad) atomicOr(&S.ctl->status, kBadIndex);
  }
}

// The changed fields of every particle, in index order, with the flag of the
// particles stepped since the last gather (cleared).
__global__ void irr_gather(State S) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.n; i += gridDim.x * blockDim.x) {
    Changed &g = S.chg[i];
    g.touched = S.touched[i];
    S.touched[i] = 0;
    if (!g.touched) continue;
    const Rec &r = S.rec[i];
    for (int d = 0; d < 3; ++d) {
      g.x[d] = r.x[d];
      g.v[d] = r.v[d];
    }
    g.t_irr = r.t;
    g.dt_irr = S.dt_irr[i];
    for (int q = 0; q < 12; ++q) {
      g.a_tot[q] = S.a_tot[12 * (size_t)i + q];
      g.a_irr[q] = S.a_irr[12 * (size_t)i + q];
    }
    g.cur_irr = S.cur_irr[i];
    g.tb_irr = S.tb_irr[i];
    g.next_irr = S.next_irr[i];
    g.new_cur_irr = S.new_cur_irr[i];
    g.lv_irr = S.lv_irr[i];
  }
}

// ------------------------------------------------------------ whole regular blocks
// The regular half of a block with the state resident here: the next block's
// particles, the j-set handed to the regular-force context, and the corrector
// and commit of every target once the context has its forces.  Each step keeps
// the host integrator's operation order (host/ac_integrator.cpp
// next_regular_block, upload_and_predict, regular_correct_one, finish_regular),
// so that a block equals the host's bit for bit.

// Sum and exclusive scan of one int per thread over a block of 256 threads.
__device__ int block_sum_int(int v) {
  __shared__ int s_part[8];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = v;
  __syncthreads();
  int r = 0;
  for (int k = 0; k < 8; ++k) r += s_part[k];
  __syncthreads();
  return r;
}

__device__ int block_exscan_int(int v) {
  __shared__ int s_warp[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  if (lane == 31) s_warp[w] = inc;
  __syncthreads();
  int before = 0;
  for (int k = 0; k < w; ++k) before += s_warp[k];
  __syncthreads();
  return before + inc - v;
}

__device__ __forceinline__ ULL reg_due(const State &S, int i) { return S.cur_reg[i] + S.tb_reg[i]; }

// next_regular_block: the smallest cur_reg + tb_reg not above block_max.
__global__ void __launch_bounds__(kThreads) blk_min(State S, ULL block_max) {
  ULL mn = ULLONG_MAX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.n; i += gridDim.x * blockDim.x) {
    const ULL t = reg_due(S, i);
    if (t <= block_max && t < mn) mn = t;
  }
  mn = block_min(mn);
  if (threadIdx.x == 0 && mn != ULLONG_MAX) atomicMin(&S.ctl->tmin, mn);
}

// Particles due at tmin per chunk of kSchedChunk.
__global__ void __launch_bounds__(kThreads) blk_count(State S) {
  const ULL t = S.ctl->tmin;
  const int b0 = blockIdx.x * kSchedChunk, b1 = min(S.n, b0 + kSchedChunk);
  int c = 0;
  for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) c += reg_due(S, i) == t;
  c = block_sum_int(c);
  if (threadIdx.x == 0) S.bcnt[blockIdx.x] = c;
}

// The particles due at tmin in ascending index: chunk b starts after the
// counts of the chunks before it, thread k of a chunk takes its 8 particles
// [8k, 8k + 8).  The last thread of the last chunk writes the total.
__global__ void __launch_bounds__(kThreads) blk_collect(State S) {
  const ULL t = S.ctl->tmin;
  int off = 0;
  for (int b = threadIdx.x; b < (int)blockIdx.x; b += blockDim.x) off += S.bcnt[b];
  off = block_sum_int(off);
  const int i0 = blockIdx.x * kSchedChunk + 8 * threadIdx.x;
  unsigned due = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q)
    if (i0 + q < S.n && reg_due(S, i0 + q) == t) due |= 1u << q;
  const int c = __popc(due);
  const int ex = block_exscan_int(c);
  int pos = off + ex;
#pragma unroll
  for (int q = 0; q < 8; ++q)
    if ((due >> q) & 1u) S.tg[pos++] = i0 + q;
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) S.ctl->m = off + ex + c;
}

// upload_and_predict's state: a0, a1 = a_tot[.][0], a_tot[.][1]; t0 = t_reg
// without neighbours, else t_irr (CalculateRegularAcceleration.cpp:371-374).
__global__ void blk_fill(State S, JsetDst d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.n; i += gridDim.x * blockDim.x) {
    const Rec &r = S.rec[i];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      d.x[3 * (size_t)i + k] = r.x[k];
      d.v[3 * (size_t)i + k] = r.v[k];
      d.a0[3 * (size_t)i + k] = S.a_tot[12 * (size_t)i + 4 * k + 0];
      d.a1[3 * (size_t)i + k] = S.a_tot[12 * (size_t)i + 4 * k + 1];
    }
    d.t0[i] = S.nnb[i] == 0 ? S.t_reg[i] : r.t;
    d.mass[i] = r.m;
    d.r2nb[i] = S.r2nb[i];
  }
}

// regular_gpu's overflow rule: r2nb *= 0.8 for every target whose list overflowed.
__global__ void blk_shrink(State S, int m, const int *nnb, int cap) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
    if (nnb[k] > cap) {
      const int i = S.tg[k];
      S.r2nb[i] = S.r2nb[i] * 0.8;
    }
}

__device__ __forceinline__ bool listed(const int *list, int n, int j) {
  for (int q = 0; q < n; ++q)
    if (list[q] == j) return true;
  return false;
}

// The host's pair_force of a changed neighbour j with sign s: j predicted to
// new_time from its own last time (t_reg without neighbours, else t_irr).
__device__ void change_terms(const State &S, int j, double new_time, double scale, double eps2,
                             const double (&pi)[3], const double (&vi)[3], double sign, double (&ta)[3],
                             double (&tj)[3]) {
  const Rec &q = S.rec[j];
  const double t0 = S.nnb[j] == 0 ? S.t_reg[j] : q.t;
  const double dt = (new_time - t0) * scale;
  double x[3], v[3], r2 = 0.0, vx = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double a0 = S.a_tot[12 * (size_t)j + 4 * d + 0], a1 = S.a_tot[12 * (size_t)j + 4 * d + 1];
    double pj, vj;
    if (dt == 0) {
      pj = q.x[d];
      vj = q.v[d];
    } else {
      pj = ((a1 * dt / 3 + a0) * dt / 2 + q.v[d]) * dt + q.x[d];
      vj = (a1 * dt / 2 + a0) * dt + q.v[d];
    }
    x[d] = pj - pi[d];
    v[d] = vj - vi[d];
    r2 += x[d] * x[d];
    vx += x[d] * v[d];
  }
  const double r2s = r2 + eps2;
  const double m_r3 = q.m / r2s / sqrt(r2s);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    ta[d] = sign * m_r3 * x[d];
    tj[d] = sign * m_r3 * (v[d] - 3 * x[d] * vx / r2s);
  }
}

// updateRegularParticleCuda (ComputeAcceleration.cpp:405-661) for the block's
// targets, one warp each, from the pre-block state: the target predicted to
// the block time (only a particle without neighbours moves), the force of
// every lost (old, not new) and gained (new, not old) neighbour in the
// interleaved order of the host's neighbour_change, the fourth-order Hermite
// corrector and the new derivatives.  Lanes compute the changed neighbours'
// terms, 32 list positions (64 slots) a round; lane c < 6 then adds component
// c in slot order: the host's sequential sums.
__global__ void __launch_bounds__(kThreads) blk_correct(State S, BlockParams B, int m, RegResults R) {
  __shared__ double s_terms[kThreads / 32][6 * 64];
  __shared__ unsigned char s_has[kThreads / 32][64];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double *terms = s_terms[wib];
  unsigned char *has = s_has[wib];
  const double scale = B.irr.scale;
  for (int k = warp; k < m; k += nwarps) {
    const int i = S.tg[k];
    // the force call is repeated until no list overflows; the clamp keeps a
    // row read inside its capacity regardless
    const int n_old = S.nnb[i], n_new = min(R.nnb[k], R.cap);
    const int *old_nb = S.nb + (size_t)i * S.cap;
    const int *new_nb = R.list + (size_t)k * R.cap;
    const Rec &r = S.rec[i];
    double at[12], ar[12], ai[12];
#pragma unroll
    for (int q = 0; q < 12; ++q) {
      at[q] = S.a_tot[12 * (size_t)i + q];
      ar[q] = S.a_reg[12 * (size_t)i + q];
      ai[q] = S.a_irr[12 * (size_t)i + q];
    }
    const double t_reg = S.t_reg[i], dt_reg = S.dt_reg[i];
    const double new_time = t_reg + dt_reg;
    const double dtp = (n_old == 0 ? dt_reg : 0.0) * scale;
    double pos[3], vel[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (dtp == 0) {
        pos[d] = r.x[d];
        vel[d] = r.v[d];
      } else {
        pos[d] = ((at[4 * d + 1] * dtp / 3 + at[4 * d + 0]) * dtp / 2 + r.v[d]) * dtp + r.x[d];
        vel[d] = (at[4 * d + 1] * dtp / 2 + at[4 * d + 0]) * dtp + r.v[d];
      }
    }
    double sum = 0.0;
    const int size = max(n_old, n_new);
    for (int base = 0; base < size; base += 32) {
      const int kk = base + lane;
      double ta[3] = {0.0, 0.0, 0.0}, tj[3] = {0.0, 0.0, 0.0};
      double ua[3] = {0.0, 0.0, 0.0}, uj[3] = {0.0, 0.0, 0.0};
      bool lost = false, gained = false;
      if (kk < n_old) {
        const int j = old_nb[kk];
        lost = !listed(new_nb, n_new, j);
        if (lost) change_terms(S, j, new_time, scale, B.irr.eps2, pos, vel, -1.0, ta, tj);
      }
      if (kk < n_new) {
        const int j = new_nb[kk];
        gained = !listed(old_nb, n_old, j);
        if (gained) change_terms(S, j, new_time, scale, B.irr.eps2, pos, vel, +1.0, ua, uj);
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        terms[d * 64 + 2 * lane] = ta[d];
        terms[(3 + d) * 64 + 2 * lane] = tj[d];
        terms[d * 64 + 2 * lane + 1] = ua[d];
        terms[(3 + d) * 64 + 2 * lane + 1] = uj[d];
      }
      has[2 * lane] = lost;
      has[2 * lane + 1] = gained;
      __syncwarp();
      if (lane < 6)
        for (int l = 0; l < 64; ++l)
          if (has[l]) sum += terms[lane * 64 + l];
      __syncwarp();
    }
    double a_tmp[3], adot_tmp[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      a_tmp[d] = __shfl_sync(0xffffffffu, sum, d);
      adot_tmp[d] = __shfl_sync(0xffffffffu, sum, 3 + d);
    }
    if (lane != 0) continue;
    // hermite_regular and commit_derivatives (ComputeAcceleration.cpp:592-660)
    const double dt = dt_reg * scale;
    const double dt2 = dt * dt, dt3 = dt2 * dt, dt4 = dt3 * dt, dt5 = dt4 * dt;
    RPend *o = &S.rpend[k];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double acc = R.acc_reg[3 * (size_t)k + d], jerk = R.jerk_reg[3 * (size_t)k + d];
      const double da_dt2 = (ar[4 * d + 0] - acc - a_tmp[d]) / dt2;
      const double adot_dt = (ar[4 * d + 1] + jerk + adot_tmp[d]) / dt;
      const double a2 = -6 * da_dt2 - 2 * adot_dt - 2 * ar[4 * d + 1] / dt;
      const double a3 = (12 * da_dt2 + 6 * adot_dt) / dt;
      o->nx[d] = pos[d] + a2 * dt4 / 24 + a3 * dt5 / 120;
      o->nv[d] = vel[d] + a2 * dt3 / 6 + a3 * dt4 / 24;
      double nr[4] = {acc, jerk, a2, a3};
      double ni[4] = {R.acc_irr[3 * (size_t)k + d], R.jerk_irr[3 * (size_t)k + d], ai[4 * d + 2], ai[4 * d + 3]};
      double nt[4] = {nr[0] + ni[0], nr[1] + ni[1], n_new == 0 ? a2 : at[4 * d + 2], n_new == 0 ? a3 : at[4 * d + 3]};
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        o->a_reg[4 * d + q] = nr[q];
        o->a_irr[4 * d + q] = ni[q];
        o->a_tot[4 * d + q] = nt[q];
      }
    }
  }
}

// calculateTimeStepReg (UpdateParticle.cpp:314-407, host/ac_integrator.cpp
// time_step_reg) with cur_reg and t_reg already advanced; lv_reg, tb_reg,
// dt_reg (and lv_irr of a particle without neighbours) updated in place.
// Returns false for a step out of range.
__device__ bool level_reg(const BlockParams &B, const double *a_reg, bool has_nb, ULL cur_reg, double t_reg,
                          int &lv_reg, ULL &tb_reg, double &dt_reg, int &lv_irr, long long &border) {
  const Params &P = B.irr;
  int lv = block_level(P, new_step_irr(a_reg, a_reg, B.eta_reg), border);
  const int lv0 = lv;
  if (lv >= lv_reg + 1) {
    if (fmod((double)cur_reg, 2.0 * (double)tb_reg) == 0 && t_reg != 0) {
      lv = lv_reg + 1;
      ULL tb = tb_reg * 2;
      // ends within lv0 - lv rounds
      while ((lv0 > lv) && (fmod((double)cur_reg, 2.0 * (double)tb) == 0)) {
        tb = 2 * tb;
        lv = lv + 1;
      }
    } else {
      lv = lv_reg;
    }
  } else if (lv < lv_reg) {
    lv = lv_reg - 1;
    if (lv0 < lv) lv--;
  } else {
    lv = lv_reg;
  }
  lv_reg = max(P.time_block, lv);
  if (!has_nb) lv_irr = lv_reg;
  dt_reg = pow2d(lv_reg);
  tb_reg = pow2_blocks(lv_reg - P.time_block);
  if (t_reg + dt_reg > 1 && t_reg != 1.0) {
    dt_reg = 1 - t_reg;
    tb_reg = B.block_max - cur_reg;
  }
  if (dt_reg * P.scale * 1e4 < 1e-9) return false;
  return !(dt_reg > 1);
}

// updateRadius (UpdateParticle.cpp:108-139, host/ac_integrator.cpp
// update_radius): the powers there are of small integers, exact in FP64, and
// are written as products.
__device__ double new_radius(double r2nb, int nnb, int fix, int nbmax) {
  if (nnb > fix) {
    const double c = (nbmax - fix);
    const double b = 0.9 / (c * c);
    const double x = nnb - fix;
    const double a = b * fabs(x) * x;
    return r2nb * (1. - a);
  }
  if (nnb < fix) {
    const double c = (nbmax - fix);
    const double b = 0.5 / (c * c * c);
    const double x = nnb - fix;
    const double a = b * (x * x * x);
    return r2nb * (1. - a);
  }
  return r2nb;
}

// RegCudaUpdate (WorkerRoutines.cpp:124-143) and finish_regular's commit, one
// warp per target: the new list, derivatives, position and velocity, then the
// regular and irregular steps, the radius and the next irregular time.
__global__ void __launch_bounds__(kThreads) blk_commit(State S, BlockParams B, int m, RegResults R) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const Params &P = B.irr;
  long long border = 0;
  for (int k = warp; k < m; k += nwarps) {
    const int i = S.tg[k];
    const int n_new = min(R.nnb[k], R.cap);
    for (int q = lane; q < n_new; q += 32) S.nb[(size_t)i * S.cap + q] = R.list[(size_t)k * R.cap + q];
    if (lane != 0) continue;
    const RPend &o = S.rpend[k];
    Rec &r = S.rec[i];
    S.nnb[i] = n_new;
#pragma unroll
    for (int q = 0; q < 12; ++q) {
      S.a_reg[12 * (size_t)i + q] = o.a_reg[q];
      S.a_irr[12 * (size_t)i + q] = o.a_irr[q];
      S.a_tot[12 * (size_t)i + q] = o.a_tot[q];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      r.x[d] = o.nx[d];
      r.v[d] = o.nv[d];
      r.a0[d] = o.a_tot[4 * d + 0];
      r.a1[d] = o.a_tot[4 * d + 1];
    }
    const ULL cur_reg = S.cur_reg[i] + S.tb_reg[i];
    const double t_reg = (double)cur_reg * P.time_step;
    int lv_reg = S.lv_reg[i], lv_irr = S.lv_irr[i];
    ULL tb_reg = S.tb_reg[i], tb_irr = S.tb_irr[i];
    double dt_reg = S.dt_reg[i], dt_irr = S.dt_irr[i];
    bool ok = level_reg(B, o.a_reg, n_new > 0, cur_reg, t_reg, lv_reg, tb_reg, dt_reg, lv_irr, border);
    // the host's time_step_irr is skipped when time_step_reg failed
    if (ok)
      ok = level_irr(P, n_new > 0, o.a_tot, o.a_irr, S.new_cur_irr[i], cur_reg, tb_reg, lv_reg, lv_irr, dt_irr,
                     tb_irr, border);
    ULL cur_irr = S.cur_irr[i];
    if (n_new == 0) {
      cur_irr = cur_reg;
      r.t = (double)cur_reg * P.time_step;
    }
    S.cur_reg[i] = cur_reg;
    S.t_reg[i] = t_reg;
    S.lv_reg[i] = lv_reg;
    S.tb_reg[i] = tb_reg;
    S.dt_reg[i] = dt_reg;
    S.lv_irr[i] = lv_irr;
    S.tb_irr[i] = tb_irr;
    S.dt_irr[i] = dt_irr;
    S.cur_irr[i] = cur_irr;
    S.r2nb[i] = new_radius(S.r2nb[i], n_new, B.fix_nb, B.nb_max);
    S.next_irr[i] = cur_irr + tb_irr;
    if (!ok) atomicOr(&S.ctl->status, kRegBad);
  }
  if (lane == 0 && border) atomicAdd((unsigned long long *)&S.ctl->borderline, (unsigned long long)border);
}

// Every particle's fields as an image (list_off = i * cap; the lists are
// copied as they lie).
__global__ void blk_gather_all(State S) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.n; i += gridDim.x * blockDim.x) {
    Image &g = S.img[i];
    const Rec &r = S.rec[i];
    for (int d = 0; d < 3; ++d) {
      g.x[d] = r.x[d];
      g.v[d] = r.v[d];
    }
    g.m = r.m;
    g.t_irr = r.t;
    g.t_reg = S.t_reg[i];
    g.dt_irr = S.dt_irr[i];
    for (int q = 0; q < 12; ++q) {
      g.a_tot[q] = S.a_tot[12 * (size_t)i + q];
      g.a_reg[q] = S.a_reg[12 * (size_t)i + q];
      g.a_irr[q] = S.a_irr[12 * (size_t)i + q];
    }
    g.cur_irr = S.cur_irr[i];
    g.tb_irr = S.tb_irr[i];
    g.next_irr = S.next_irr[i];
    g.new_cur_irr = S.new_cur_irr[i];
    g.cur_reg = S.cur_reg[i];
    g.tb_reg = S.tb_reg[i];
    g.r2nb = S.r2nb[i];
    g.dt_reg = S.dt_reg[i];
    g.lv_irr = S.lv_irr[i];
    g.lv_reg = S.lv_reg[i];
    g.nnb = S.nnb[i];
    g.index = i;
    g.list_off = (long long)i * S.cap;
  }
}

template <class T>
cudaError_t dalloc(T **p, size_t count) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  return cudaMalloc((void **)p, std::max<size_t>(count, 1) * sizeof(T));
}

}  // namespace

struct Engine {
  int device = 0;
  int sm_count = 148;
  int max_grid = 0;  // co-resident blocks of irr_levels
  cudaStream_t stream = nullptr;
  std::string err;
  int n = 0, cap = 0;
  int alloc_n = 0;  // particles the arrays and the pinned staging hold
  State S{};
  Image *h_img = nullptr;  // pinned
  int *h_lists = nullptr;  // pinned
  Changed *h_chg = nullptr;  // pinned
  // pinned control words, one way each: a copy from pageable memory waits in
  // the driver's staging path, which the host threads of many engines share
  Ctl *h_ctl_in = nullptr, *h_ctl_out = nullptr;
  // how a call waits for its stream: < 0 the stream synchronisation (the
  // thread keeps its core), else poll for spin_us then sleep in a blocking
  // event wait (many engines driven from more host threads than cores)
  int spin_us = -1;
  cudaEvent_t ev_wait = nullptr;
};

namespace {

int fail(Engine *e, int code, const std::string &msg) {
  e->err = msg;
  return code;
}

#define ECK(call, what)                                                                    \
  do {                                                                                     \
    cudaError_t err_ = (call);                                                             \
    if (err_ != cudaSuccess)                                                               \
      return fail(e, err_ == cudaErrorMemoryAllocation ? ABYSS_ERR_OOM : ABYSS_ERR_CUDA,   \
                  std::string(what) + ": " + cudaGetErrorString(err_));                    \
  } while (0)

void free_state(State &S) {
  void *ps[] = {S.rec, S.a_tot, S.a_reg, S.a_irr, S.t_reg, S.dt_irr, S.cur_irr, S.tb_irr, S.next_irr,
                S.new_cur_irr, S.cur_reg, S.tb_reg, S.lv_irr, S.lv_reg, S.nnb, S.nb, S.touched, S.members, S.pend,
                S.img, S.lists, S.chg, S.r2nb, S.dt_reg, S.tg, S.bcnt, S.rpend};
  for (void *p : ps)
    if (p) cudaFree(p);
  Ctl *c = S.ctl;
  S = State{};
  S.ctl = c;
}

// The control words reset on `s` (tmin to its largest value).  The previous
// copy out of the pinned word has finished: every engine call waits for its
// stream before it returns.
int reset_ctl(Engine *e, cudaStream_t s) {
  Ctl c{};
  c.tmin = ULLONG_MAX;
  c.lmin[0] = c.lmin[1] = ULLONG_MAX;
  *e->h_ctl_in = c;
  ECK(cudaMemcpyAsync(e->S.ctl, e->h_ctl_in, sizeof(Ctl), cudaMemcpyHostToDevice, s), "reset control words");
  return ABYSS_OK;
}
int reset_ctl(Engine *e) { return reset_ctl(e, e->stream); }

// Wait on the host for everything queued on `s`, by the engine's policy.
cudaError_t sync_stream(Engine *e, cudaStream_t s) {
  if (e->spin_us < 0 || !e->ev_wait) return cudaStreamSynchronize(s);
  cudaError_t err = cudaEventRecord(e->ev_wait, s);
  if (err != cudaSuccess) return err;
  const auto t0 = std::chrono::steady_clock::now();
  const auto spin = std::chrono::microseconds(e->spin_us);
  for (;;) {
    err = cudaEventQuery(e->ev_wait);
    if (err != cudaErrorNotReady) return err;
    if (std::chrono::steady_clock::now() - t0 >= spin) break;
  }
  return cudaEventSynchronize(e->ev_wait);
}

int read_ctl(Engine *e, Ctl *c, cudaStream_t s) {
  ECK(cudaMemcpyAsync(e->h_ctl_out, e->S.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s), "read control words");
  ECK(sync_stream(e, s), "synchronize");
  *c = *e->h_ctl_out;
  return ABYSS_OK;
}
int read_ctl(Engine *e, Ctl *c) { return read_ctl(e, c, e->stream); }

}  // namespace

int engine_create(int device, Engine **out) {
  if (!out) return ABYSS_ERR_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    return ABYSS_ERR_NODEVICE;
  }
  Engine *e = new Engine;
  e->device = device;
  cudaSetDevice(device);
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || !prop.cooperativeLaunch) {
    delete e;
    return ABYSS_ERR_NODEVICE;
  }
  e->sm_count = prop.multiProcessorCount;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, irr_levels, kThreads, 0) != cudaSuccess || per_sm < 1 ||
      cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc((void **)&e->S.ctl, sizeof(Ctl)) != cudaSuccess ||
      cudaHostAlloc((void **)&e->h_ctl_in, sizeof(Ctl), cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc((void **)&e->h_ctl_out, sizeof(Ctl), cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    engine_destroy(e);
    return ABYSS_ERR_CUDA;
  }
  e->max_grid = per_sm * e->sm_count;
  *out = e;
  return ABYSS_OK;
}

void engine_destroy(Engine *e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->stream) cudaStreamSynchronize(e->stream);
  free_state(e->S);
  if (e->S.ctl) cudaFree(e->S.ctl);
  if (e->h_img) cudaFreeHost(e->h_img);
  if (e->h_lists) cudaFreeHost(e->h_lists);
  if (e->h_chg) cudaFreeHost(e->h_chg);
  if (e->h_ctl_in) cudaFreeHost(e->h_ctl_in);
  if (e->h_ctl_out) cudaFreeHost(e->h_ctl_out);
  if (e->ev_wait) cudaEventDestroy(e->ev_wait);
  if (e->stream) cudaStreamDestroy(e->stream);
  delete e;
}

const char *engine_error(const Engine *e) { return e ? e->err.c_str() : "null engine"; }

int engine_set_wait(Engine *e, int spin_us) {
  if (!e) return ABYSS_ERR_ARG;
  if (spin_us >= 0 && !e->ev_wait) {
    cudaSetDevice(e->device);
    ECK(cudaEventCreateWithFlags(&e->ev_wait, cudaEventBlockingSync | cudaEventDisableTiming), "wait event");
  }
  e->spin_us = spin_us < 0 ? -1 : spin_us;
  return ABYSS_OK;
}

namespace {
constexpr size_t kPoolMax = 16;  // engines kept per process
std::mutex g_pool_mu;
std::vector<Engine *> g_pool;
}  // namespace

int engine_take(int device, Engine **out) {
  if (!out) return ABYSS_ERR_ARG;
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    for (size_t k = g_pool.size(); k-- > 0;)
      if (g_pool[k]->device == device) {
        *out = g_pool[k];
        g_pool.erase(g_pool.begin() + (long)k);
        (*out)->err.clear();
        return ABYSS_OK;
      }
  }
  return engine_create(device, out);
}

void engine_give(Engine *e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (cudaStreamSynchronize(e->stream) == cudaSuccess) {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (g_pool.size() < kPoolMax) {
      g_pool.push_back(e);
      return;
    }
  }
  cudaGetLastError();
  engine_destroy(e);
}

int engine_reserve(Engine *e, int n, int cap) {
  if (!e || n <= 0 || cap <= 0) return ABYSS_ERR_ARG;
  if (n == e->n && cap == e->cap) return ABYSS_OK;
  cudaSetDevice(e->device);
  ECK(cudaStreamSynchronize(e->stream), "synchronize");
  if (cap == e->cap && n <= e->alloc_n) {
    // a smaller (or regrown) cluster in the arrays already held: no
    // allocation, which would synchronize the device for every other stream
    ECK(cudaMemsetAsync(e->S.touched, 0, sizeof(int) * (size_t)n, e->stream), "clear");
    ECK(cudaMemsetAsync(e->S.nnb, 0, sizeof(int) * (size_t)n, e->stream), "clear");
    ECK(cudaStreamSynchronize(e->stream), "synchronize");
    e->S.n = n;
    e->n = n;
    return ABYSS_OK;
  }
  // growth by at least half again, so that an engine reused for clusters of
  // rising sizes reallocates only a few times
  const int grow = cap == e->cap ? e->alloc_n + e->alloc_n / 2 : 0;
  const int n_alloc = std::max(n, grow);
  free_state(e->S);
  if (e->h_img) cudaFreeHost(e->h_img);
  if (e->h_lists) cudaFreeHost(e->h_lists);
  if (e->h_chg) cudaFreeHost(e->h_chg);
  e->h_img = nullptr;
  e->h_lists = nullptr;
  e->h_chg = nullptr;
  e->n = e->cap = e->alloc_n = 0;
  State &S = e->S;
  const size_t N = n_alloc;
  ECK(dalloc(&S.rec, N), "alloc");
  ECK(dalloc(&S.a_tot, 12 * N), "alloc");
  ECK(dalloc(&S.a_reg, 12 * N), "alloc");
  ECK(dalloc(&S.a_irr, 12 * N), "alloc");
  ECK(dalloc(&S.t_reg, N), "alloc");
  ECK(dalloc(&S.dt_irr, N), "alloc");
  ECK(dalloc(&S.cur_irr, N), "alloc");
  ECK(dalloc(&S.tb_irr, N), "alloc");
  ECK(dalloc(&S.next_irr, N), "alloc");
  ECK(dalloc(&S.new_cur_irr, N), "alloc");
  ECK(dalloc(&S.cur_reg, N), "alloc");
  ECK(dalloc(&S.tb_reg, N), "alloc");
  ECK(dalloc(&S.lv_irr, N), "alloc");
  ECK(dalloc(&S.lv_reg, N), "alloc");
  ECK(dalloc(&S.nnb, N), "alloc");
  ECK(dalloc(&S.nb, N * cap), "alloc");
  ECK(dalloc(&S.touched, N), "alloc");
  ECK(dalloc(&S.members, N), "alloc");
  ECK(dalloc(&S.pend, N), "alloc");
  ECK(dalloc(&S.img, N), "alloc");
  ECK(dalloc(&S.lists, N * cap), "alloc");
  ECK(dalloc(&S.chg, N), "alloc");
  ECK(dalloc(&S.r2nb, N), "alloc");
  ECK(dalloc(&S.dt_reg, N), "alloc");
  ECK(dalloc(&S.tg, N), "alloc");
  ECK(dalloc(&S.bcnt, N / kSchedChunk + 1), "alloc");
  ECK(dalloc(&S.rpend, N), "alloc");
  ECK(cudaMemsetAsync(S.touched, 0, sizeof(int) * N, e->stream), "clear");
  ECK(cudaMemsetAsync(S.nnb, 0, sizeof(int) * N, e->stream), "clear");
  ECK(cudaHostAlloc((void **)&e->h_img, sizeof(Image) * N, cudaHostAllocDefault), "pinned images");
  ECK(cudaHostAlloc((void **)&e->h_lists, sizeof(int) * N * cap, cudaHostAllocDefault), "pinned lists");
  ECK(cudaHostAlloc((void **)&e->h_chg, sizeof(Changed) * N, cudaHostAllocDefault), "pinned changes");
  S.n = n;
  S.cap = cap;
  e->n = n;
  e->cap = cap;
  e->alloc_n = n_alloc;
  return ABYSS_OK;
}

Image *engine_images(Engine *e) { return e ? e->h_img : nullptr; }
Changed *engine_changed(Engine *e) { return e ? e->h_chg : nullptr; }
int *engine_lists(Engine *e) { return e ? e->h_lists : nullptr; }

int engine_upload(Engine *e, int count, long long list_entries) {
  if (!e || count < 0 || count > e->n || list_entries < 0 || list_entries > (long long)e->n * e->cap)
    return ABYSS_ERR_ARG;
  if (count == 0) return ABYSS_OK;
  cudaSetDevice(e->device);
  int rc = reset_ctl(e);
  if (rc != ABYSS_OK) return rc;
  for (int k = 0; k < count; ++k) {
    const Image &g = e->h_img[k];
    if (g.nnb < 0 || g.list_off < 0 || g.list_off + g.nnb > list_entries)
      return fail(e, ABYSS_ERR_ARG, "upload: an image's list lies outside the staged lists");
  }
  ECK(cudaMemcpyAsync(e->S.img, e->h_img, sizeof(Image) * (size_t)count, cudaMemcpyHostToDevice, e->stream),
      "H2D images");
  if (list_entries > 0)
    ECK(cudaMemcpyAsync(e->S.lists, e->h_lists, sizeof(int) * (size_t)list_entries, cudaMemcpyHostToDevice,
                        e->stream),
        "H2D lists");
  const int blocks = std::max(1, std::min((count + 255) / 256, 4 * e->sm_count));
  irr_scatter<<<blocks, 256, 0, e->stream>>>(e->S, count);
  ECK(cudaGetLastError(), "scatter launch");
  Ctl c;
  rc = read_ctl(e, &c);
  if (rc != ABYSS_OK) return rc;
  if (c.status & kBadIndex) return fail(e, ABYSS_ERR_ARG, "upload: an image names a particle outside the cluster");
  return ABYSS_OK;
}

int engine_run_levels(Engine *e, const Params &p, RunStats *st, void *stream) {
  if (!e || e->n <= 0) return ABYSS_ERR_ARG;
  cudaSetDevice(e->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : e->stream;
  int rc = reset_ctl(e, s);
  if (rc != ABYSS_OK) return rc;
  // one block per SM at most (a level's barrier waits on every block), and
  // enough blocks that a slice fits the block's member list
  int grid = std::max(1, std::min(e->sm_count, (e->n + 127) / 128));
  grid = std::max(grid, (e->n + kMaxSlice - 1) / kMaxSlice);
  if (grid > e->max_grid) return fail(e, ABYSS_ERR_ARG, "level loop: cluster too large for one co-resident grid");
  int slice = (e->n + grid - 1) / grid;
  State S = e->S;
  Params P = p;
  void *args[] = {&S, &P, &slice};
  ECK(cudaLaunchCooperativeKernel((const void *)irr_levels, dim3(grid), dim3(kThreads), args, 0, s),
      "level loop launch");
  Ctl c;
  rc = read_ctl(e, &c, s);
  if (rc != ABYSS_OK) return rc;
  if (st) {
    st->levels = c.levels;
    st->steps = c.steps;
    st->borderline = c.borderline;
    for (int q = 0; q < 6; ++q) st->cycles[q] = c.cycles[q];
  }
  if (c.status & kTimeout) return fail(e, ABYSS_ERR_TIMEOUT, "level loop: a grid barrier wait ran out");
  if (c.status & kBad) return fail(e, ABYSS_ERR_STATE, "irregular time step out of range");
  return ABYSS_OK;
}

int engine_download(Engine *e) {
  if (!e || e->n <= 0) return ABYSS_ERR_ARG;
  cudaSetDevice(e->device);
  const int blocks = std::max(1, std::min((e->n + 255) / 256, 4 * e->sm_count));
  irr_gather<<<blocks, 256, 0, e->stream>>>(e->S);
  ECK(cudaGetLastError(), "gather launch");
  ECK(cudaMemcpyAsync(e->h_chg, e->S.chg, sizeof(Changed) * (size_t)e->n, cudaMemcpyDeviceToHost, e->stream),
      "D2H changes");
  ECK(sync_stream(e, e->stream), "synchronize");
  return ABYSS_OK;
}

int engine_steps(Engine *e, const Params &p, int count, const int *idx, double *new_pos, double *new_vel,
                 double *a_irr, double *a_tot, int *lv_irr, double *dt_irr, ULL *tb_irr) {
  if (!e || e->n <= 0 || count < 0 || (count > 0 && !idx)) return ABYSS_ERR_ARG;
  if (count == 0) return ABYSS_OK;
  for (int k = 0; k < count; ++k)
    if (idx[k] < 0 || idx[k] >= e->n) return fail(e, ABYSS_ERR_ARG, "steps: index outside the cluster");
  cudaSetDevice(e->device);
  int rc = reset_ctl(e);
  if (rc != ABYSS_OK) return rc;
  int *d_idx = nullptr, *d_lv = nullptr;
  double *d_pos = nullptr, *d_vel = nullptr, *d_ai = nullptr, *d_at = nullptr, *d_dt = nullptr;
  ULL *d_tb = nullptr;
  const size_t K = count;
  cudaError_t err = cudaSuccess;
  if (err == cudaSuccess) err = cudaMalloc((void **)&d_idx, 4 * K);
  if (err == cudaSuccess) err = cudaMalloc((void **)&d_lv, 4 * K);
  if (err == cudaSuccess) err = cudaMalloc((void **)&d_pos, 24 * K);
  if (err == cudaSuccess) err = cudaMalloc((void **)&d_vel, 24 * K);
  if (err == cudaSuccess) err = cudaMalloc((void **)&d_ai, 96 * K);
  if (err == cudaSuccess) err = cudaMalloc((void **)&d_at, 96 * K);
  if (err == cudaSuccess) err = cudaMalloc((void **)&d_dt, 8 * K);
  if (err == cudaSuccess) err = cudaMalloc((void **)&d_tb, 8 * K);
  if (err == cudaSuccess) err = cudaMemcpyAsync(d_idx, idx, 4 * K, cudaMemcpyHostToDevice, e->stream);
  if (err == cudaSuccess) {
    const int blocks = std::max(1, std::min((int)((K * 32 + kThreads - 1) / kThreads), 8 * e->sm_count));
    irr_steps<<<blocks, kThreads, 0, e->stream>>>(e->S, p, count, d_idx, d_pos, d_vel, d_ai, d_at, d_lv, d_dt, d_tb);
    err = cudaGetLastError();
  }
  struct Out {
    void *dst;
    const void *src;
    size_t bytes;
  } outs[] = {{new_pos, d_pos, 24 * K}, {new_vel, d_vel, 24 * K}, {a_irr, d_ai, 96 * K}, {a_tot, d_at, 96 * K},
              {lv_irr, d_lv, 4 * K},     {dt_irr, d_dt, 8 * K},   {tb_irr, d_tb, 8 * K}};
  for (const Out &o : outs)
    if (err == cudaSuccess && o.dst) err = cudaMemcpyAsync(o.dst, o.src, o.bytes, cudaMemcpyDeviceToHost, e->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
  void *ps[] = {d_idx, d_lv, d_pos, d_vel, d_ai, d_at, d_dt, d_tb};
  for (void *q : ps)
    if (q) cudaFree(q);
  if (err != cudaSuccess) return fail(e, ABYSS_ERR_CUDA, std::string("steps: ") + cudaGetErrorString(err));
  Ctl c;
  rc = read_ctl(e, &c);
  if (rc != ABYSS_OK) return rc;
  if (c.status & kBad) return fail(e, ABYSS_ERR_STATE, "irregular time step out of range");
  return ABYSS_OK;
}

// ------------------------------------------------------------ whole regular blocks

const int *engine_block_targets(const Engine *e) { return e ? e->S.tg : nullptr; }

int engine_next_block(Engine *e, void *stream, ULL block_max, ULL *tmin, int *m) {
  if (!e || e->n <= 0 || !tmin || !m) return ABYSS_ERR_ARG;
  cudaSetDevice(e->device);
  cudaStream_t s = (cudaStream_t)stream;
  int rc = reset_ctl(e, s);
  if (rc != ABYSS_OK) return rc;
  const int chunks = (e->n + kSchedChunk - 1) / kSchedChunk;
  const int blocks = std::max(1, std::min((e->n + kThreads - 1) / kThreads, 4 * e->sm_count));
  blk_min<<<blocks, kThreads, 0, s>>>(e->S, block_max);
  blk_count<<<chunks, kThreads, 0, s>>>(e->S);
  blk_collect<<<chunks, kThreads, 0, s>>>(e->S);
  ECK(cudaGetLastError(), "next block launch");
  Ctl c;
  rc = read_ctl(e, &c, s);
  if (rc != ABYSS_OK) return rc;
  if (c.tmin == ULLONG_MAX) {
    *tmin = block_max;
    *m = 0;
  } else {
    *tmin = c.tmin;
    *m = c.m;
  }
  return ABYSS_OK;
}

int engine_fill_jset(Engine *e, void *stream, const JsetDst &d) {
  if (!e || e->n <= 0 || !d.x || !d.v || !d.a0 || !d.a1 || !d.t0 || !d.mass || !d.r2nb) return ABYSS_ERR_ARG;
  cudaSetDevice(e->device);
  const int blocks = std::max(1, std::min((e->n + 255) / 256, 4 * e->sm_count));
  blk_fill<<<blocks, 256, 0, (cudaStream_t)stream>>>(e->S, d);
  ECK(cudaGetLastError(), "j-set fill launch");
  return ABYSS_OK;
}

int engine_shrink_radii(Engine *e, void *stream, int m, const int *nnb, int cap) {
  if (!e || m < 0 || m > e->n || (m > 0 && !nnb)) return ABYSS_ERR_ARG;
  if (m == 0) return ABYSS_OK;
  cudaSetDevice(e->device);
  const int blocks = std::max(1, std::min((m + 255) / 256, 4 * e->sm_count));
  blk_shrink<<<blocks, 256, 0, (cudaStream_t)stream>>>(e->S, m, nnb, cap);
  ECK(cudaGetLastError(), "radius launch");
  return ABYSS_OK;
}

int engine_correct_block(Engine *e, void *stream, const BlockParams &bp, int m, const RegResults &r,
                         long long *borderline) {
  if (!e || m <= 0 || m > e->n || !r.acc_reg || !r.jerk_reg || !r.acc_irr || !r.jerk_irr || !r.nnb || !r.list)
    return ABYSS_ERR_ARG;
  if (r.cap > e->cap || bp.nb_max != e->cap)
    return fail(e, ABYSS_ERR_ARG, "regular block: list capacity differs from the engine's");
  cudaSetDevice(e->device);
  cudaStream_t s = (cudaStream_t)stream;
  int rc = reset_ctl(e, s);
  if (rc != ABYSS_OK) return rc;
  const int blocks = std::max(1, std::min((int)(((size_t)m * 32 + kThreads - 1) / kThreads), 8 * e->sm_count));
  blk_correct<<<blocks, kThreads, 0, s>>>(e->S, bp, m, r);
  blk_commit<<<blocks, kThreads, 0, s>>>(e->S, bp, m, r);
  ECK(cudaGetLastError(), "corrector launch");
  Ctl c;
  rc = read_ctl(e, &c, s);
  if (rc != ABYSS_OK) return rc;
  if (borderline) *borderline += c.borderline;
  if (c.status & kRegBad) return fail(e, ABYSS_ERR_STATE, "regular time step out of range");
  return ABYSS_OK;
}

int engine_download_all(Engine *e) {
  if (!e || e->n <= 0) return ABYSS_ERR_ARG;
  cudaSetDevice(e->device);
  const int blocks = std::max(1, std::min((e->n + 255) / 256, 4 * e->sm_count));
  blk_gather_all<<<blocks, 256, 0, e->stream>>>(e->S);
  ECK(cudaGetLastError(), "gather launch");
  ECK(cudaMemcpyAsync(e->h_img, e->S.img, sizeof(Image) * (size_t)e->n, cudaMemcpyDeviceToHost, e->stream),
      "D2H images");
  ECK(cudaMemcpyAsync(e->h_lists, e->S.nb, sizeof(int) * (size_t)e->n * e->cap, cudaMemcpyDeviceToHost, e->stream),
      "D2H lists");
  ECK(sync_stream(e, e->stream), "synchronize");
  return ABYSS_OK;
}


}  // namespace abyss_irr
