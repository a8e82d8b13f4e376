// Host Ahmad-Cohen integrator (include/abyss_ac.h).
//
// Single-process restatement of the reference's block-timestep loop with the
// GPU regular force behind the C ABI:
//   initialisation  RootRoutines.cpp:104-330 (InitAcc1, InitAcc2, InitTime,
//                   time-step correction, time_block)
//   main loop       RootRoutines.cpp:448-1075: next regular block
//                   (updateNextRegTime, :1310-1338), irregular levels in
//                   increasing NextBlockIrr (skip list, :488-1005), then the
//                   regular step (calculateRegAccelerationOnGPU + RegCudaUpdate)
//   per particle    ComputeAcceleration.cpp:14-190 (irregular),
//                   :405-661 (regular corrector after the GPU force),
//                   UpdateParticle.cpp:13-407 (predictor, radius, time steps),
//                   TimeStepRoutines.cpp:10-115, Initialize.cpp:16-230.
// Deliberate differences, each for a reason stated at the site:
//   * softening eps2 in all force terms (the configurations ask for it);
//   * separate eta for regular and irregular steps;
//   * the irregular corrector's dt^5 is dt^4 * dt (the reference reads an
//     uninitialised dt5 at ComputeAcceleration.cpp:162, line 120 commented out);
//   * two-phase blocks: every particle of a block is computed from the
//     pre-block state before any is committed (the reference's workers
//     overwrite a_tot while others still predict from it);
//   * a target whose list overflows nb_max has its radius shrunk and the
//     regular call re-run, instead of a device assert.
// The same loop can run with its irregular levels on the GPU
// (abyss_ac_set_device_irregular, irregular.cu) or with whole blocks there and
// the state kept on the device (abyss_ac_set_device_resident: resident_block
// below); both give the host loop's results bit for bit.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <condition_variable>
#include <deque>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <mutex>
#include <thread>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_set>
#include <vector>

#include <cuda_runtime.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../../../include/abyss_ac.h"
#include "../../../include/abyss_ens.h"
#include "../../../include/abyss_io.h"
#include "../../../include/abyss_irr.h"
#include "../../../include/abyss_reg.h"
#include "../irregular.h"
#include "../ctx_internal.h"
#include "pair_terms.h"

namespace {

typedef unsigned long long ULL;


double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct alignas(64) Star {
  // what a neighbour's irregular step reads: x, v, m, t_irr on one cache line,
  // a_tot[.][0..1] on the next two
  double x[3], v[3], m, t_irr = 0;
  double a_tot[3][4], a_reg[3][4], a_irr[3][4];
  std::vector<int> nb;
  double r2nb;
  double t_reg = 0, dt_reg = 0, dt_irr = 0;
  ULL cur_reg = 0, cur_irr = 0, new_cur_irr = 0, next_irr = 0, tb_reg = 0, tb_irr = 0;
  int lv_reg = 0, lv_irr = 0;
};

// Result of one particle's block computation, committed in phase two.
struct Pending {
  double new_x[3], new_v[3];
  double a_tot[3][4], a_reg[3][4], a_irr[3][4];
  std::vector<int> new_nb;
  bool move = false;
  // irregular step bookkeeping (calculateTimeStepIrr results)
  int lv_irr = 0;
  double dt_irr = 0;
  ULL tb_irr = 0, new_cur_irr = 0;
};

using abyss_host::NbRec;

}  // namespace

struct abyss_ac {
  abyss_ctx *ctx = nullptr;
  abyss_ac_params p{};
  std::vector<Star> s;
  int n = 0;
  double scale = 1.0;  // EnzoTimeStep
  int time_block = -30;
  ULL block_max = 1ull << 30;
  double time_step = std::ldexp(1.0, -30);
  ULL next_reg_block = 0;
  bool done = false;
  std::string err;
  abyss_ac_stats st{};
  // last regular call
  std::vector<int> last_targets, last_nnb, last_list;
  std::vector<double> last_px, last_pv, last_r2, last_acc, last_jerk;
  int last_cap = 0;
  std::vector<double> reg_airr, reg_jirr;  // buffers of the regular call's FP64 irregular part
  // split form: the regular block begun and not yet ended
  bool in_block = false;
  std::vector<int> block_targets;
  // the neighbour fields mirrored in Morton order of the particles' positions
  // (slot[i] is particle i's record), so that a particle's neighbours, which
  // are near it in space, are near in memory too
  std::vector<NbRec> jrec;
  std::vector<int> slot;
  // irregular levels on the device (abyss_ac_set_device_irregular): the
  // engine's copy of the state is current when eng_synced, except for the
  // particles in eng_dirty (committed by the host since the last download)
  bool dev_irr = false;
  abyss_irr::Engine *eng = nullptr;
  bool eng_synced = false;
  std::vector<int> eng_dirty;
  long long dev_borderline = 0;
  long long dev_cycles[6] = {0, 0, 0, 0, 0, 0};
  double dev_sec_copy = 0.0;
  // whole blocks on the device (abyss_ac_set_device_resident): the engine's
  // state is the state of record while dev_res; the particles here are a copy,
  // refreshed from the device when host_stale and something reads them
  bool dev_res = false, host_stale = false;
  long long res_borderline = 0;
  double res_sec_sync = 0.0;
  int res_last_m = 0;  // the last device block's size (its record is the context's)
  // pinned staging of the j-set uploaded for each regular block: x, v, a0, a1
  // ([n][3] each), t0, m, r2nb ([n] each)
  double *jstage = nullptr;
  size_t jstage_n = 0;
  // wall seconds outside the stats' timers: j-set fill, upload and prediction;
  // the next-block scan
  double sec_jset = 0.0, sec_sched = 0.0;
  ~abyss_ac() {
    if (eng) abyss_irr::engine_give(eng);
    if (jstage) cudaFreeHost(jstage);
  }
};

namespace {

// 2^e and 2^e as a block count, exactly what the reference's
// static_cast<double>(pow(2, e)) and static_cast<ULL>(pow(2, e)) give for every
// int e (ldexp is exact; the libm pow call is not needed).
inline double pow2(int e) { return std::ldexp(1.0, e); }
inline ULL pow2_blocks(int e) { return static_cast<ULL>(std::ldexp(1.0, e)); }

// UpdateParticle.cpp:37-59.
inline void predict(const Star &p, double dt_code, double scale, double pos[3], double vel[3]) {
  const double dt = dt_code * scale;
  for (int d = 0; d < 3; ++d) {
    if (dt == 0) {
      pos[d] = p.x[d];
      vel[d] = p.v[d];
    } else {
      pos[d] = ((p.a_tot[d][1] * dt / 3 + p.a_tot[d][0]) * dt / 2 + p.v[d]) * dt + p.x[d];
      vel[d] = (p.a_tot[d][1] * dt / 2 + p.a_tot[d][0]) * dt + p.v[d];
    }
  }
}

// TimeStepRoutines.cpp:10-25 (eta passed in).
double new_step_reg(const double df[3][4], double eta) {
  const double F2 = df[0][0] * df[0][0] + df[1][0] * df[1][0] + df[2][0] * df[2][0];
  const double Fdot2 = df[0][1] * df[0][1] + df[1][1] * df[1][1] + df[2][1] * df[2][1];
  const double F2dot2 = df[0][2] * df[0][2] + df[1][2] * df[1][2] + df[2][2] * df[2][2];
  const double F3dot2 = df[0][3] * df[0][3] + df[1][3] * df[1][3] + df[2][3] * df[2][3];
  double dta = (std::sqrt(F2 * F2dot2) + Fdot2) / (std::sqrt(Fdot2 * F3dot2) + F2dot2);
  return std::sqrt(eta * dta);
}

// TimeStepRoutines.cpp:28-63 and :65-100 (same formula).
double new_step_irr(const double f[3][4], const double df[3][4], double eta) {
  const double F2 = f[0][0] * f[0][0] + f[1][0] * f[1][0] + f[2][0] * f[2][0];
  const double Fdot2 = df[0][1] * df[0][1] + df[1][1] * df[1][1] + df[2][1] * df[2][1];
  const double F2dot2 = df[0][2] * df[0][2] + df[1][2] * df[1][2] + df[2][2] * df[2][2];
  const double F3dot2 = df[0][3] * df[0][3] + df[1][3] * df[1][3] + df[2][3] * df[2][3];
  double ts = (std::sqrt(F2 * F2dot2) + Fdot2) / (std::sqrt(Fdot2 * F3dot2) + F2dot2);
  return std::sqrt(eta * ts);
}

// TimeStepRoutines.cpp:102-115.
void block_step(const abyss_ac *ac, double dt, int &level, ULL &block, double &step) {
  level = static_cast<int>(std::floor(std::log(dt / ac->scale) / std::log(2.0)));
  if (level < ac->time_block) level = ac->time_block;
  step = pow2(level);
  block = pow2_blocks(level - ac->time_block);
}

// UpdateParticle.cpp:151-241 (calculateTimeStepIrr).
// The irregular step of a particle from its fields (a_tot, a_irr are the
// particle's new derivatives); lv_irr, dt_irr, tb_irr are updated in place.
void time_step_irr_of(const abyss_ac *ac, bool has_nb, const double (&a_tot)[3][4], const double (&a_irr)[3][4],
                      ULL new_cur_irr, ULL cur_reg, ULL tb_reg, int lv_reg, int &lv_irr, double &dt_irr,
                      ULL &tb_irr);

void time_step_irr(const abyss_ac *ac, Star &p) {
  time_step_irr_of(ac, !p.nb.empty(), p.a_tot, p.a_irr, p.new_cur_irr, p.cur_reg, p.tb_reg, p.lv_reg, p.lv_irr,
                   p.dt_irr, p.tb_irr);
}

void time_step_irr_of(const abyss_ac *ac, bool has_nb, const double (&a_tot)[3][4], const double (&a_irr)[3][4],
                      ULL new_cur_irr, ULL cur_reg, ULL tb_reg, int lv_reg, int &lv_irr, double &dt_irr,
                      ULL &tb_irr) {
  struct {
    ULL new_cur_irr, cur_reg, tb_reg, tb_irr;
    int lv_reg, lv_irr;
    double dt_irr;
  } p{new_cur_irr, cur_reg, tb_reg, tb_irr, lv_reg, lv_irr, dt_irr};
  if (!has_nb) {
    lv_irr = p.lv_reg;
    dt_irr = pow2(p.lv_reg);
    tb_irr = pow2_blocks(p.lv_reg - ac->time_block);
    return;
  }
  int lv;
  ULL tb;
  double stp;
  block_step(ac, new_step_irr(a_tot, a_irr, ac->p.eta_irr), lv, tb, stp);
  if (lv > p.lv_irr) {
    if (std::fmod((double)p.new_cur_irr, 2.0 * (double)p.tb_irr) == 0) {
      lv = p.lv_irr + 1;
      tb = 2 * p.tb_irr;
    } else {
      lv = p.lv_irr;
      tb = p.tb_irr;
    }
  } else if (lv < p.lv_irr) {
    if (lv < p.lv_irr - 1) {
      lv = p.lv_irr - 2;
      tb = p.tb_irr / 4;
    } else {
      lv = p.lv_irr - 1;
      tb = p.tb_irr / 2;
    }
  } else {
    lv = p.lv_irr;
    tb = p.tb_irr;
  }
  const ULL reg_end = p.cur_reg + p.tb_reg;
  while (((p.new_cur_irr < reg_end) && (p.new_cur_irr + tb > reg_end)) || (lv >= p.lv_reg)) {
    lv--;
    tb = (ULL)(tb * 0.5);
  }
  lv_irr = std::max(ac->time_block, lv);
  dt_irr = pow2(lv_irr);
  tb_irr = pow2_blocks(lv_irr - ac->time_block);
  if (dt_irr > 1) throw std::runtime_error("irregular time step exceeds the run");
}

// UpdateParticle.cpp:314-407 (calculateTimeStepReg).
void time_step_reg(const abyss_ac *ac, Star &p) {
  int lv;
  ULL tb;
  double stp;
  block_step(ac, new_step_reg(p.a_reg, ac->p.eta_reg), lv, tb, stp);
  const int lv0 = lv;
  if (lv >= p.lv_reg + 1) {
    if (std::fmod((double)p.cur_reg, 2.0 * (double)p.tb_reg) == 0 && p.t_reg != 0) {
      lv = p.lv_reg + 1;
      tb = p.tb_reg * 2;
      while ((lv0 > lv) && (std::fmod((double)p.cur_reg, 2.0 * (double)tb) == 0)) {
        tb = 2 * tb;
        lv = lv + 1;
      }
    } else {
      lv = p.lv_reg;
    }
  } else if (lv < p.lv_reg) {
    lv = p.lv_reg - 1;
    if (lv0 < lv) lv--;
  } else {
    lv = p.lv_reg;
  }
  p.lv_reg = std::max(ac->time_block, lv);
  if (p.nb.empty()) p.lv_irr = p.lv_reg;
  p.dt_reg = pow2(p.lv_reg);
  p.tb_reg = pow2_blocks(p.lv_reg - ac->time_block);
  if (p.t_reg + p.dt_reg > 1 && p.t_reg != 1.0) {
    p.dt_reg = 1 - p.t_reg;
    p.tb_reg = ac->block_max - p.cur_reg;
  }
  if (p.dt_reg * ac->scale * 1e4 < 1e-9) throw std::runtime_error("regular time step is too small");
  if (p.dt_reg > 1) throw std::runtime_error("regular time step exceeds the run");
}

// UpdateParticle.cpp:108-139 (updateRadius), FixNumNeighbor/NumNeighborMax as parameters.
void update_radius(const abyss_ac *ac, Star &p) {
  const int nnb = (int)p.nb.size();
  const int fix = ac->p.fix_nb, nbmax = ac->p.nb_max;
  if (nnb > fix) {
    const int n = 2;
    const double c = (nbmax - fix);
    const double b = 0.9 / std::pow(c, n);
    const double x = nnb - fix;
    const double a = n % 2 == 0 ? b * std::abs(x) * std::pow(x, n - 1) : b * std::pow(x, n);
    p.r2nb *= (1. - a);
  } else if (nnb < fix) {
    const int n = 3;
    const double c = (nbmax - fix);
    const double b = 0.5 / std::pow(c, n);
    const double x = nnb - fix;
    const double a = n % 2 == 0 ? b * std::abs(x) * std::pow(x, n - 1) : b * std::pow(x, n);
    p.r2nb *= (1. - a);
  }
}

// Force of j on i (predicted pos/vel of both), softened.
inline void pair_force(const double pi[3], const double vi[3], const double pj[3], const double vj[3],
                       double mj, double eps2, double a[3], double ad[3], double sign) {
  double x[3], v[3], r2 = 0.0, vx = 0.0;
  for (int d = 0; d < 3; ++d) {
    x[d] = pj[d] - pi[d];
    v[d] = vj[d] - vi[d];
    r2 += x[d] * x[d];
    vx += x[d] * v[d];
  }
  const double r2s = r2 + eps2;
  const double m_r3 = mj / r2s / std::sqrt(r2s);
  for (int d = 0; d < 3; ++d) {
    a[d] += sign * m_r3 * x[d];
    ad[d] += sign * m_r3 * (v[d] - 3 * x[d] * vx / r2s);
  }
}

int set_threads(const abyss_ac *ac) {
#ifdef _OPENMP
  if (ac->p.threads > 0) omp_set_num_threads(ac->p.threads);
  return omp_get_max_threads();
#else
  (void)ac;
  return 1;
#endif
}

// One GPU regular-force call over `targets` with the j-set already predicted on
// the device.  Overflowing targets get r2nb *= 0.8 and the call is repeated.
int regular_gpu(abyss_ac *ac, const std::vector<int> &targets, bool upload_r2,
                std::vector<double> &acc, std::vector<double> &jerk, std::vector<double> &airr,
                std::vector<double> &jirr, std::vector<int> &nnb, std::vector<int> &lst) {
  const int m = (int)targets.size();
  const int cap = ac->p.nb_max;
  // every element is written by the call below: sized, not cleared (the list
  // alone is m x cap ints, tens of MB per block at N = 65 536)
  acc.resize(3 * (size_t)m);
  jerk.resize(3 * (size_t)m);
  airr.resize(3 * (size_t)m);
  jirr.resize(3 * (size_t)m);
  nnb.resize(m);
  lst.resize((size_t)m * cap);
  (void)upload_r2;
  for (int attempt = 0; attempt < 40; ++attempt) {
    int ovf = 0;
    const double t0 = now_s();
    int rc = abyss_regular_force(ac->ctx, m, targets.data(), ac->p.eps2, cap, nullptr, acc.data(),
                                 jerk.data(), airr.data(), jirr.data(), nnb.data(), lst.data(), &ovf);
    ac->st.sec_reg_gpu += now_s() - t0;
    if (rc < 0) {
      ac->err = std::string("regular force: ") + abyss_last_error(ac->ctx);
      return rc;
    }
    if (rc != ABYSS_WARN_OVERFLOW) return ABYSS_OK;
    // shrink the radius of every overflowing target and re-upload the j-set radii
    ac->st.radius_retries++;
    for (int k = 0; k < m; ++k)
      if (nnb[k] > cap) ac->s[targets[k]].r2nb *= 0.8;
    return 2;  // caller re-predicts and retries
  }
  ac->err = "regular force: neighbour lists kept overflowing";
  return ABYSS_ERR_STATE;
}

int upload_and_predict(abyss_ac *ac, double new_time) {
  const double tstart = now_s();
  const int n = ac->n;
  const size_t N = n;
  // the staging is pinned (plain DMA, no driver staging) and kept across blocks
  if (ac->jstage_n != N) {
    if (ac->jstage) cudaFreeHost(ac->jstage);
    ac->jstage = nullptr;
    ac->jstage_n = 0;
    if (cudaHostAlloc((void **)&ac->jstage, sizeof(double) * 15 * N, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      ac->jstage = nullptr;
      ac->err = "upload/predict: pinned staging allocation failed";
      return ABYSS_ERR_OOM;
    }
    ac->jstage_n = N;
  }
  double *x = ac->jstage, *v = x + 3 * N, *a0 = v + 3 * N, *a1 = a0 + 3 * N, *t0 = a1 + 3 * N, *m = t0 + N,
         *r2 = m + N;
#pragma omp parallel for schedule(static) if (n >= 8192)
  for (int j = 0; j < n; ++j) {
    const Star &p = ac->s[j];
    for (int d = 0; d < 3; ++d) {
      x[3 * (size_t)j + d] = p.x[d];
      v[3 * (size_t)j + d] = p.v[d];
      a0[3 * (size_t)j + d] = p.a_tot[d][0];
      a1[3 * (size_t)j + d] = p.a_tot[d][1];
    }
    // CalculateRegularAcceleration.cpp:371-374
    t0[j] = p.nb.empty() ? p.t_reg : p.t_irr;
    m[j] = p.m;
    r2[j] = p.r2nb;
  }
  int rc = abyss_upload_state(ac->ctx, n, x, v, a0, a1, t0, m, r2);
  ac->last_r2.assign(r2, r2 + N);
  if (rc == ABYSS_OK) rc = abyss_predict(ac->ctx, new_time, ac->scale);
  if (rc == ABYSS_OK) rc = abyss_synchronize(ac->ctx);
  if (rc != ABYSS_OK) ac->err = std::string("upload/predict: ") + abyss_last_error(ac->ctx);
  ac->sec_jset += now_s() - tstart;
  return rc;
}

// Initialize.cpp:102-185 (CalculateAcceleration23) with softened r^2, for all i,
// on the device (abyss_init_derivs23: the same sequential FP64 sums, bit for bit).
int init_acc23(abyss_ac *ac) {
  const int n = ac->n;
  std::vector<double> x(3 * (size_t)n), v(3 * (size_t)n), m(n), r2(n), a0(3 * (size_t)n), a1(3 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    const Star &p = ac->s[i];
    for (int d = 0; d < 3; ++d) {
      x[3 * (size_t)i + d] = p.x[d];
      v[3 * (size_t)i + d] = p.v[d];
      a0[3 * (size_t)i + d] = p.a_tot[d][0];
      a1[3 * (size_t)i + d] = p.a_tot[d][1];
    }
    m[i] = p.m;
    r2[i] = p.r2nb;
  }
  std::vector<double> reg2(3 * (size_t)n), reg3(3 * (size_t)n), irr2(3 * (size_t)n), irr3(3 * (size_t)n);
  const int rc = abyss_init_derivs23(ac->ctx, n, x.data(), v.data(), m.data(), r2.data(), a0.data(), a1.data(),
                                     ac->p.eps2, reg2.data(), reg3.data(), irr2.data(), irr3.data());
  if (rc != ABYSS_OK) {
    ac->err = std::string("init_derivs23: ") + abyss_last_error(ac->ctx);
    return rc;
  }
  for (int i = 0; i < n; ++i) {
    Star &p = ac->s[i];
    for (int d = 0; d < 3; ++d) {
      const size_t k = 3 * (size_t)i + d;
      p.a_reg[d][2] = reg2[k];
      p.a_reg[d][3] = reg3[k];
      p.a_irr[d][2] = irr2[k];
      p.a_irr[d][3] = irr3[k];
      p.a_tot[d][2] = p.a_reg[d][2] + p.a_irr[d][2];
      p.a_tot[d][3] = p.a_reg[d][3] + p.a_irr[d][3];
    }
  }
  return ABYSS_OK;
}

// Initialize.cpp:199-230 (initializeTimeStep).
void init_time_step(abyss_ac *ac, Star &p) {
  double stp;
  block_step(ac, new_step_irr(p.a_reg, p.a_reg, ac->p.eta_reg), p.lv_reg, p.tb_reg, stp);
  p.dt_reg = std::min(1.0, stp);
  p.tb_reg = std::min(ac->block_max, p.tb_reg);
  p.lv_reg = std::min(0, p.lv_reg);
  if (!p.nb.empty()) {
    block_step(ac, new_step_irr(p.a_tot, p.a_irr, ac->p.eta_irr), p.lv_irr, p.tb_irr, p.dt_irr);
  } else {
    p.tb_irr = p.tb_reg;
    p.lv_irr = p.lv_reg;
    p.dt_irr = p.dt_reg;
  }
  p.t_irr = p.t_reg = 0;
  p.cur_irr = p.cur_reg = 0;
}

int initialise(abyss_ac *ac, const double *r2nb) {
  const double t0 = now_s();
  const int n = ac->n;
  set_threads(ac);
  // InitAcc1: FP64-split acc and jerk at t = 0 on the GPU (CalculateAcceleration01,
  // Initialize.cpp:16-92, uses r2 > R2 for the regular part; the regular-step rule
  // r2 < R2 is used here so that lists agree with every later regular step).
  std::vector<int> all(n);
  for (int i = 0; i < n; ++i) {
    all[i] = i;
    ac->s[i].r2nb = r2nb[i];
  }
  std::vector<double> acc, jerk, airr, jirr;
  std::vector<int> nnb, lst;
  for (int attempt = 0;; ++attempt) {
    int rc = upload_and_predict(ac, 0.0);
    if (rc != ABYSS_OK) return rc;
    rc = regular_gpu(ac, all, true, acc, jerk, airr, jirr, nnb, lst);
    if (rc == ABYSS_OK) break;
    if (rc != 2 || attempt > 40) return rc < 0 ? rc : ABYSS_ERR_STATE;
  }
  const int cap = ac->p.nb_max;
  for (int i = 0; i < n; ++i) {
    Star &p = ac->s[i];
    for (int d = 0; d < 3; ++d) {
      for (int o = 0; o < 4; ++o) p.a_reg[d][o] = p.a_irr[d][o] = p.a_tot[d][o] = 0.0;
      p.a_reg[d][0] = acc[3 * (size_t)i + d];
      p.a_reg[d][1] = jerk[3 * (size_t)i + d];
      p.a_irr[d][0] = airr[3 * (size_t)i + d];
      p.a_irr[d][1] = jirr[3 * (size_t)i + d];
      p.a_tot[d][0] = p.a_reg[d][0] + p.a_irr[d][0];
      p.a_tot[d][1] = p.a_reg[d][1] + p.a_irr[d][1];
    }
    p.nb.assign(lst.begin() + (size_t)i * cap, lst.begin() + (size_t)i * cap + nnb[i]);
  }
  {  // InitAcc2
    const int rc = init_acc23(ac);
    if (rc != ABYSS_OK) return rc;
  }
  for (int i = 0; i < n; ++i) init_time_step(ac, ac->s[i]);  // InitTime
  // time-step correction and time_block (RootRoutines.cpp:240-270)
  int min_level = 0;
  for (int i = 0; i < n; ++i) {
    Star &p = ac->s[i];
    if (!p.nb.empty())
      while (p.lv_irr >= p.lv_reg) {
        p.dt_irr *= 0.5;
        p.tb_irr = (ULL)(p.tb_irr * 0.5);
        p.lv_irr--;
      }
    min_level = std::min(min_level, p.lv_irr);
  }
  ac->time_block = std::max(-60, min_level - 30);  // MIN_LEVEL_BUFFER, def.h:33
  ac->block_max = pow2_blocks(-ac->time_block);
  ac->time_step = pow2(ac->time_block);
  for (int i = 0; i < n; ++i) {
    Star &p = ac->s[i];
    p.tb_irr = pow2_blocks(p.lv_irr - ac->time_block);
    p.tb_reg = pow2_blocks(p.lv_reg - ac->time_block);
    p.next_irr = p.cur_irr + p.tb_irr;
  }
  ac->next_reg_block = 0;
  ac->st.sec_init += now_s() - t0;
  return ABYSS_OK;
}

// ComputeAcceleration.cpp:14-190 for one particle, into `out` (phase one).
void irregular_one(const abyss_ac *ac, int i, Pending &out) {
  // an irregular step commits a_tot and a_irr (never a_reg); both are written
  // in full below unless the particle has no neighbours
  const Star &p = ac->s[i];
  if (p.nb.empty()) {
    std::memcpy(out.a_tot, p.a_tot, sizeof(out.a_tot));
    std::memcpy(out.a_irr, p.a_irr, sizeof(out.a_irr));
    out.move = false;
    return;
  }
  out.move = true;
  const double new_time = p.t_irr + p.dt_irr;
  const double dt = p.dt_irr * ac->scale;
  double pos[3], vel[3], a_tmp[3] = {0, 0, 0}, adot_tmp[3] = {0, 0, 0};
  predict(p, p.dt_irr, ac->scale, pos, vel);
  // the neighbours' state gathered, their terms computed independently (SIMD),
  // then added in neighbour order: the same sums as the one-pass loop
  const int nn = (int)p.nb.size();
  // the records are fetched ahead of the terms, which gather them themselves
  const NbRec *J = ac->jrec.data();
  const int *sl = ac->slot.data();
  for (int k = 0; k < nn; ++k) {
    const char *q = reinterpret_cast<const char *>(&J[sl[p.nb[k]]]);
    __builtin_prefetch(q);
    __builtin_prefetch(q + 64);
  }
  thread_local std::vector<double> ta, tj;
  ta.resize(3 * (size_t)nn);
  tj.resize(3 * (size_t)nn);
  abyss_host::irregular_terms(nn, p.nb.data(), sl, J, pos, vel, new_time, ac->scale, ac->p.eps2, ta.data(),
                              tj.data());
  for (int k = 0; k < nn; ++k)
    for (int d = 0; d < 3; ++d) {
      a_tmp[d] += ta[3 * k + d];
      adot_tmp[d] += tj[3 * k + d];
    }
  const double dt_ex = (new_time - p.t_reg) * ac->scale;
  const double dt2 = dt * dt, dt3 = dt2 * dt, dt4 = dt3 * dt, dt5 = dt4 * dt;
  for (int d = 0; d < 3; ++d) {
    const double da_dt2 = (p.a_irr[d][0] - a_tmp[d]) / dt2;
    const double adot_dt = (p.a_irr[d][1] + adot_tmp[d]) / dt;
    const double a2 = -6 * da_dt2 - 2 * adot_dt - 2 * p.a_irr[d][1] / dt;
    const double a3 = (12 * da_dt2 + 6 * adot_dt) / dt;
    out.new_x[d] = pos[d] + a2 * dt4 / 24 + a3 * dt5 / 120;
    out.new_v[d] = vel[d] + a2 * dt3 / 6 + a3 * dt4 / 24;
    out.a_irr[d][0] = a_tmp[d];
    out.a_irr[d][1] = adot_tmp[d];
    out.a_irr[d][2] = a2;
    out.a_irr[d][3] = a3;
  }
  for (int d = 0; d < 3; ++d) {
    out.a_tot[d][0] = p.a_reg[d][0] + out.a_irr[d][0] + p.a_reg[d][1] * dt_ex;
    out.a_tot[d][1] = p.a_reg[d][1] + out.a_irr[d][1];
    out.a_tot[d][2] = p.a_reg[d][2] + out.a_irr[d][2];
    out.a_tot[d][3] = p.a_reg[d][3] + out.a_irr[d][3];
  }
}

void put_rec(abyss_ac *ac, int i) {
  const Star &p = ac->s[i];
  NbRec &r = ac->jrec[ac->slot[i]];
  for (int d = 0; d < 3; ++d) {
    r.x[d] = p.x[d];
    r.v[d] = p.v[d];
    r.a0[d] = p.a_tot[d][0];
    r.a1[d] = p.a_tot[d][1];
  }
  r.m = p.m;
  r.t = p.t_irr;
}

// Morton order (21 bits per axis over the bounding box) of the positions now.
void build_slots(abyss_ac *ac) {
  const int n = ac->n;
  double lo[3] = {HUGE_VAL, HUGE_VAL, HUGE_VAL}, hi[3] = {-HUGE_VAL, -HUGE_VAL, -HUGE_VAL};
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], ac->s[i].x[d]);
      hi[d] = std::max(hi[d], ac->s[i].x[d]);
    }
  auto spread = [](ULL v) {
    v &= 0x1fffffULL;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
  };
  std::vector<std::pair<ULL, int>> key(n);
  for (int i = 0; i < n; ++i) {
    ULL c[3];
    for (int d = 0; d < 3; ++d) {
      const double w = hi[d] > lo[d] ? (ac->s[i].x[d] - lo[d]) / (hi[d] - lo[d]) : 0.0;
      c[d] = (ULL)(std::min(std::max(w, 0.0), 1.0) * 2097151.0);
    }
    key[i] = {spread(c[0]) | spread(c[1]) << 1 | spread(c[2]) << 2, i};
  }
  std::sort(key.begin(), key.end());
  ac->slot.assign(n, 0);
  for (int r = 0; r < n; ++r) ac->slot[key[r].second] = r;
  ac->jrec.assign(n, NbRec{});
}

// A thread's share of the particles filed under their next irregular level,
// grouped by level.  A level's particles go to few next levels, so a linear
// search over the groups is enough.
struct Filing {
  std::vector<std::pair<ULL, std::vector<int>>> groups;
  void add(ULL key, int i) {
    for (auto &g : groups)
      if (g.first == key) {
        g.second.push_back(i);
        return;
      }
    groups.emplace_back(key, std::vector<int>{i});
  }
  void drain_into(std::map<ULL, std::vector<int>> &levels) {
    for (auto &g : groups) {
      std::vector<int> &dst = levels[g.first];
      dst.insert(dst.end(), g.second.begin(), g.second.end());
    }
    groups.clear();
  }
};

// One irregular level: every particle's step from the pre-level state, then
// (after the loop's barrier) every commit.  The loops are work-shared among the
// threads of the enclosing parallel region, or run by the caller alone outside
// one.  *bad is set when a step fails; nothing is committed then.
void run_level(abyss_ac *ac, const std::vector<int> &P, std::vector<Pending> &pend, std::vector<Filing> &filing,
               int *bad) {
  const int np = (int)P.size();
#pragma omp for schedule(dynamic, 8)
  for (int k = 0; k < np; ++k) {
    irregular_one(ac, P[k], pend[k]);
    // NewCurrentBlockIrr and the new irregular step use this particle's new
    // derivatives (WorkerRoutines.cpp:46-64), without touching its state.
    const Star &sp = ac->s[P[k]];
    int lv_irr = sp.lv_irr;
    double dt_irr = sp.dt_irr;
    ULL tb_irr = sp.tb_irr;
    const ULL new_cur = sp.cur_irr + sp.tb_irr;
    try {
      time_step_irr_of(ac, !sp.nb.empty(), pend[k].a_tot, pend[k].a_irr, new_cur, sp.cur_reg, sp.tb_reg, sp.lv_reg,
                       lv_irr, dt_irr, tb_irr);
    } catch (const std::exception &) {
#pragma omp atomic write
      *bad = 1;
    }
    pend[k].lv_irr = lv_irr;
    pend[k].dt_irr = dt_irr;
    pend[k].tb_irr = tb_irr;
    pend[k].new_cur_irr = new_cur;
  }
  // the loop's barrier: every step is done and *bad final
  int failed;
#pragma omp atomic read
  failed = *bad;
  if (failed) return;
  // phase two: commit (IrrForce results + IrrUpdate, WorkerRoutines.cpp:76-87)
#pragma omp for schedule(static)
  for (int k = 0; k < np; ++k) {
    Star &p = ac->s[P[k]];
    const Pending &q = pend[k];
    p.lv_irr = q.lv_irr;
    p.dt_irr = q.dt_irr;
    p.tb_irr = q.tb_irr;
    p.new_cur_irr = q.new_cur_irr;
    std::memcpy(p.a_tot, q.a_tot, sizeof(p.a_tot));
    std::memcpy(p.a_irr, q.a_irr, sizeof(p.a_irr));
    p.next_irr = p.new_cur_irr + p.tb_irr;
    if (!p.nb.empty() && q.move) {
      for (int d = 0; d < 3; ++d) {
        p.x[d] = q.new_x[d];
        p.v[d] = q.new_v[d];
      }
    }
    p.cur_irr = p.new_cur_irr;
    p.t_irr = p.cur_irr * ac->time_step;
    put_rec(ac, P[k]);
    // filed under its next level by the committing thread
    if (p.next_irr <= ac->next_reg_block) {
#ifdef _OPENMP
      filing[omp_get_thread_num()].add(p.next_irr, P[k]);
#else
      filing[0].add(p.next_irr, P[k]);
#endif
    }
  }
}

// The integrator's fields of a particle as the device irregular phase takes
// them; its list goes to lists[list_off ..].
void pack_image(const abyss_ac *ac, int i, abyss_irr::Image &g, int *lists, long long list_off) {
  const Star &p = ac->s[i];
  for (int d = 0; d < 3; ++d) {
    g.x[d] = p.x[d];
    g.v[d] = p.v[d];
  }
  g.m = p.m;
  g.t_irr = p.t_irr;
  g.t_reg = p.t_reg;
  g.dt_irr = p.dt_irr;
  std::memcpy(g.a_tot, p.a_tot, sizeof(g.a_tot));
  std::memcpy(g.a_reg, p.a_reg, sizeof(g.a_reg));
  std::memcpy(g.a_irr, p.a_irr, sizeof(g.a_irr));
  g.cur_irr = p.cur_irr;
  g.tb_irr = p.tb_irr;
  g.next_irr = p.next_irr;
  g.new_cur_irr = p.new_cur_irr;
  g.cur_reg = p.cur_reg;
  g.tb_reg = p.tb_reg;
  g.lv_irr = p.lv_irr;
  g.lv_reg = p.lv_reg;
  g.nnb = (int)p.nb.size();
  g.index = i;
  g.list_off = list_off;
  g.r2nb = p.r2nb;
  g.dt_reg = p.dt_reg;
  if (!p.nb.empty()) std::memcpy(lists + list_off, p.nb.data(), sizeof(int) * p.nb.size());
}

// What an irregular phase changed, back into particle i's fields.
void unpack_changed(abyss_ac *ac, int i, const abyss_irr::Changed &g) {
  Star &p = ac->s[i];
  for (int d = 0; d < 3; ++d) {
    p.x[d] = g.x[d];
    p.v[d] = g.v[d];
  }
  p.t_irr = g.t_irr;
  p.dt_irr = g.dt_irr;
  std::memcpy(p.a_tot, g.a_tot, sizeof(p.a_tot));
  std::memcpy(p.a_irr, g.a_irr, sizeof(p.a_irr));
  p.cur_irr = g.cur_irr;
  p.tb_irr = g.tb_irr;
  p.next_irr = g.next_irr;
  p.new_cur_irr = g.new_cur_irr;
  p.lv_irr = g.lv_irr;
}

// The irregular levels up to the next regular block on the device
// (irregular.cu): the particles the host changed since the last call go up,
// the level loop runs on the GPU, every particle's irregular fields come back.
int irregular_levels_device(abyss_ac *ac) {
  const double t0 = now_s();
  using namespace abyss_irr;
  int rc = ABYSS_OK;
  if (!ac->eng) {
    rc = engine_take(abyss::ctx_device(ac->ctx), &ac->eng);
    if (rc != ABYSS_OK) {
      ac->err = "device irregular steps: no engine on the context's device";
      return rc;
    }
    ac->eng_synced = false;
  }
  engine_set_wait(ac->eng, abyss::ctx_wait_spin(ac->ctx));  // the context's wait policy
  const int n = ac->n, cap = ac->p.nb_max;
  for (int i = 0; i < n; ++i)
    if ((int)ac->s[i].nb.size() > cap) {
      ac->err = "device irregular steps: a neighbour list longer than nb_max";
      return ABYSS_ERR_STATE;
    }
  rc = engine_reserve(ac->eng, n, cap);
  if (rc != ABYSS_OK) {
    ac->err = engine_error(ac->eng);
    ac->eng_synced = false;
    return rc;
  }
  Image *img = engine_images(ac->eng);
  int *lists = engine_lists(ac->eng);
  // the particles to send: all of them, or those the host committed since
  std::vector<int> &dirty = ac->eng_dirty;
  if (!ac->eng_synced) {
    dirty.resize(n);
    for (int i = 0; i < n; ++i) dirty[i] = i;
  } else {
    std::sort(dirty.begin(), dirty.end());
    dirty.erase(std::unique(dirty.begin(), dirty.end()), dirty.end());
  }
  const int count = (int)dirty.size();
  std::vector<long long> off(count + 1, 0);
  for (int k = 0; k < count; ++k) off[k + 1] = off[k] + (long long)ac->s[dirty[k]].nb.size();
#pragma omp parallel for schedule(static) if (count >= 16384)
  for (int k = 0; k < count; ++k) pack_image(ac, dirty[k], img[k], lists, off[k]);
  rc = engine_upload(ac->eng, count, off[count]);
  if (rc != ABYSS_OK) {
    ac->err = engine_error(ac->eng);
    ac->eng_synced = false;
    return rc;
  }
  ac->eng_dirty.clear();
  const double t1 = now_s();
  Params P;
  P.scale = ac->scale;
  P.time_step = ac->time_step;
  P.eps2 = ac->p.eps2;
  P.eta_irr = ac->p.eta_irr;
  P.ln2 = std::log(2.0);
  P.time_block = ac->time_block;
  P.next_reg_block = ac->next_reg_block;
  RunStats rs;
  const int run = engine_run_levels(ac->eng, P, &rs);
  const double t2 = now_s();
  // the levels committed before a failure are kept, as on the host
  rc = engine_download(ac->eng);
  if (rc != ABYSS_OK) {
    ac->err = engine_error(ac->eng);
    ac->eng_synced = false;
    return rc;
  }
  const Changed *chg = engine_changed(ac->eng);
#pragma omp parallel for schedule(static) if (n >= 16384)
  for (int i = 0; i < n; ++i)
    if (chg[i].touched) unpack_changed(ac, i, chg[i]);
  ac->eng_synced = true;
  ac->st.irr_levels += rs.levels;
  ac->st.irr_steps += rs.steps;
  ac->dev_borderline += rs.borderline;
  for (int q = 0; q < 6; ++q) ac->dev_cycles[q] += rs.cycles[q];
  const double t3 = now_s();
  ac->dev_sec_copy += (t1 - t0) + (t3 - t2);
  ac->st.sec_irr += t3 - t0;
  if (run != ABYSS_OK) {
    ac->err = engine_error(ac->eng);
    return run;
  }
  return ABYSS_OK;
}

// ------------------------------------------------------------ whole blocks on the device
// With abyss_ac_set_device_resident the state of record lives in the engine's
// device arrays and a block never leaves the GPU: the next block's particles
// (updateNextRegTime), the irregular levels, the j-set handed to the context,
// the regular force and the corrector, commit, time steps and radii
// (irregular.cu blk_*).  The host learns the block time and size and reads
// the particles back only when something asks for them.

// Every field of particle i from a device image (and its list).
void unpack_image(abyss_ac *ac, int i, const abyss_irr::Image &g, const int *list) {
  Star &p = ac->s[i];
  for (int d = 0; d < 3; ++d) {
    p.x[d] = g.x[d];
    p.v[d] = g.v[d];
  }
  p.m = g.m;
  p.t_irr = g.t_irr;
  p.t_reg = g.t_reg;
  p.dt_irr = g.dt_irr;
  p.dt_reg = g.dt_reg;
  p.r2nb = g.r2nb;
  std::memcpy(p.a_tot, g.a_tot, sizeof(p.a_tot));
  std::memcpy(p.a_reg, g.a_reg, sizeof(p.a_reg));
  std::memcpy(p.a_irr, g.a_irr, sizeof(p.a_irr));
  p.cur_irr = g.cur_irr;
  p.tb_irr = g.tb_irr;
  p.next_irr = g.next_irr;
  p.new_cur_irr = g.new_cur_irr;
  p.cur_reg = g.cur_reg;
  p.tb_reg = g.tb_reg;
  p.lv_irr = g.lv_irr;
  p.lv_reg = g.lv_reg;
  p.nb.assign(list, list + g.nnb);
}

// The particles here from the device, if a device block changed them since
// they were last read.  Logically const: the copy is a cache of the device's.
int resident_sync_host(const abyss_ac *cac) {
  abyss_ac *ac = const_cast<abyss_ac *>(cac);
  if (!ac->dev_res || !ac->host_stale) return ABYSS_OK;
  const double t0 = now_s();
  int rc = abyss_irr::engine_download_all(ac->eng);
  if (rc != ABYSS_OK) {
    ac->err = std::string("device state: ") + abyss_irr::engine_error(ac->eng);
    return rc;
  }
  const abyss_irr::Image *img = abyss_irr::engine_images(ac->eng);
  const int *lists = abyss_irr::engine_lists(ac->eng);
  const size_t cap = ac->p.nb_max;
  int failed = 0;
#pragma omp parallel for schedule(static) reduction(+ : failed) if (ac->n >= 16384)
  for (int i = 0; i < ac->n; ++i) {
    try {
      unpack_image(ac, i, img[i], lists + (size_t)i * cap);
    } catch (const std::bad_alloc &) {
      failed++;
    }
  }
  if (failed) {
    ac->err = "device state: host allocation failed";
    return ABYSS_ERR_OOM;
  }
  ac->host_stale = false;
  ac->res_sec_sync += now_s() - t0;
  return ABYSS_OK;
}

// The engine holds every particle (after the mode was switched on).
int resident_ensure(abyss_ac *ac) {
  using namespace abyss_irr;
  if (!ac->eng) {
    int rc = engine_take(abyss::ctx_device(ac->ctx), &ac->eng);
    if (rc != ABYSS_OK) {
      ac->err = "device blocks: no engine on the context's device";
      return rc;
    }
    ac->eng_synced = false;
  }
  engine_set_wait(ac->eng, abyss::ctx_wait_spin(ac->ctx));  // the context's wait policy
  if (ac->eng_synced) return ABYSS_OK;
  const double t0 = now_s();
  const int n = ac->n, cap = ac->p.nb_max;
  for (int i = 0; i < n; ++i)
    if ((int)ac->s[i].nb.size() > cap) {
      ac->err = "device blocks: a neighbour list longer than nb_max";
      return ABYSS_ERR_STATE;
    }
  int rc = engine_reserve(ac->eng, n, cap);
  if (rc != ABYSS_OK) {
    ac->err = engine_error(ac->eng);
    return rc;
  }
  Image *img = engine_images(ac->eng);
  int *lists = engine_lists(ac->eng);
  std::vector<long long> off(n + 1, 0);
  for (int i = 0; i < n; ++i) off[i + 1] = off[i] + (long long)ac->s[i].nb.size();
#pragma omp parallel for schedule(static) if (n >= 16384)
  for (int i = 0; i < n; ++i) pack_image(ac, i, img[i], lists, off[i]);
  rc = engine_upload(ac->eng, n, off[n]);
  if (rc != ABYSS_OK) {
    ac->err = engine_error(ac->eng);
    return rc;
  }
  ac->eng_synced = true;
  ac->eng_dirty.clear();
  ac->res_sec_sync += now_s() - t0;
  return ABYSS_OK;
}

abyss_irr::Params irr_params(const abyss_ac *ac) {
  abyss_irr::Params P;
  P.scale = ac->scale;
  P.time_step = ac->time_step;
  P.eps2 = ac->p.eps2;
  P.eta_irr = ac->p.eta_irr;
  P.ln2 = std::log(2.0);
  P.time_block = ac->time_block;
  P.next_reg_block = ac->next_reg_block;
  return P;
}

// One block with the state on the device: the same steps, in the same order,
// as next_regular_block + irregular_levels + regular_block.
int resident_block(abyss_ac *ac) {
  using namespace abyss_irr;
  int rc = resident_ensure(ac);
  if (rc != ABYSS_OK) return rc;
  Engine *e = ac->eng;
  void *stream = abyss_stream(ac->ctx);
  const int n = ac->n, cap = ac->p.nb_max;
  double t0 = now_s();
  ULL tmin = 0;
  int m = 0;
  rc = engine_next_block(e, stream, ac->block_max, &tmin, &m);
  ac->sec_sched += now_s() - t0;
  if (rc != ABYSS_OK) {
    ac->err = std::string("device blocks: ") + engine_error(e);
    return rc;
  }
  ac->next_reg_block = tmin;
  if (m <= 0) {
    ac->err = "device blocks: no particle due before the end of the run";
    return ABYSS_ERR_STATE;
  }
  // the irregular levels up to the block
  t0 = now_s();
  Params P = irr_params(ac);
  RunStats rs;
  ac->host_stale = true;
  const int run = engine_run_levels(e, P, &rs, stream);  // the context's stream: one stream per integration
  ac->st.irr_levels += rs.levels;
  ac->st.irr_steps += rs.steps;
  ac->dev_borderline += rs.borderline;
  for (int q = 0; q < 6; ++q) ac->dev_cycles[q] += rs.cycles[q];
  ac->st.sec_irr += now_s() - t0;
  if (run != ABYSS_OK) {
    ac->err = engine_error(e);
    return run;
  }
  // the regular force; a target whose list overflowed has its radius shrunk
  // and the call is repeated (regular_gpu)
  const double new_time = ac->next_reg_block * ac->time_step;
  for (int attempt = 0;; ++attempt) {
    t0 = now_s();
    JsetDst d{};
    rc = abyss::ctx_state_buffers(ac->ctx, n, &d);
    if (rc == ABYSS_OK) rc = engine_fill_jset(e, stream, d);
    if (rc == ABYSS_OK) rc = abyss_predict(ac->ctx, new_time, ac->scale);
    ac->sec_jset += now_s() - t0;
    t0 = now_s();
    if (rc == ABYSS_OK) rc = abyss::ctx_targets_from_device(ac->ctx, m, engine_block_targets(e));
    if (rc == ABYSS_OK) rc = abyss_launch(ac->ctx, ac->p.eps2, cap, nullptr);
    int st = ABYSS_OK, ovf = 0;
    if (rc == ABYSS_OK) rc = abyss::ctx_launch_status(ac->ctx, &st, &ovf);
    ac->st.sec_reg_gpu += now_s() - t0;
    if (rc == ABYSS_OK) rc = st;
    if (rc != ABYSS_OK) {
      ac->err = std::string("regular force: ") + abyss_last_error(ac->ctx);
      return rc;
    }
    if (ovf == 0) break;
    if (attempt > 40) {
      ac->err = "regular force: neighbour lists kept overflowing";
      return ABYSS_ERR_STATE;
    }
    ac->st.radius_retries++;
    RegResults r{};
    rc = abyss::ctx_results(ac->ctx, &r);
    if (rc == ABYSS_OK) rc = engine_shrink_radii(e, stream, m, r.nnb, cap);
    if (rc != ABYSS_OK) {
      ac->err = std::string("device blocks: ") + engine_error(e);
      return rc;
    }
  }
  // corrector, commit, time steps and radii
  t0 = now_s();
  BlockParams bp;
  bp.irr = P;
  bp.eta_reg = ac->p.eta_reg;
  bp.block_max = ac->block_max;
  bp.fix_nb = ac->p.fix_nb;
  bp.nb_max = cap;
  RegResults r{};
  rc = abyss::ctx_results(ac->ctx, &r);
  ac->res_last_m = 0;
  ac->st.pairs += (double)m * n;
  if (rc == ABYSS_OK) rc = engine_correct_block(e, stream, bp, m, r, &ac->res_borderline);
  ac->st.sec_reg_host += now_s() - t0;
  if (rc != ABYSS_OK) {
    ac->err = engine_error(e);
    return rc;
  }
  ac->res_last_m = m;
  ac->st.reg_steps += m;
  ac->st.blocks++;
  return ABYSS_OK;
}

// abyss_ac_last_regular of a device block: the record is the context's last
// launch (targets, radii and predicted j-set as the force saw them).
int resident_last_regular(const abyss_ac *ac, int *m, int *targets, double *px, double *pv, double *r2nb,
                          double *acc_reg, double *jerk_reg, int *nnb, int *list, int list_cap) {
  const int mm = ac->res_last_m;
  *m = 0;
  if (mm <= 0) return ABYSS_ERR_STATE;
  if (!targets && !px && !pv && !r2nb && !acc_reg && !jerk_reg && !nnb && !list) {
    *m = mm;  // the size alone
    return ABYSS_OK;
  }
  const size_t M = mm, cap = ac->p.nb_max;
  std::vector<double> acc(3 * M), jerk(3 * M);
  std::vector<int> nn(M), lst(M * cap);
  int ovf = 0;
  int rc = abyss_fetch(ac->ctx, acc.data(), jerk.data(), nullptr, nullptr, nn.data(), lst.data(), &ovf);
  if (rc == ABYSS_OK) rc = abyss::ctx_read_targets(ac->ctx, targets, r2nb);
  if (rc == ABYSS_OK && (px || pv)) rc = abyss_read_predicted(ac->ctx, px, pv, nullptr);
  if (rc != ABYSS_OK) return rc;
  *m = mm;
  for (size_t k = 0; k < M; ++k) {
    for (int d = 0; d < 3; ++d) {
      if (acc_reg) acc_reg[3 * k + d] = acc[3 * k + d];
      if (jerk_reg) jerk_reg[3 * k + d] = jerk[3 * k + d];
    }
    if (nnb) nnb[k] = nn[k];
    if (list)
      for (size_t q = 0; q < std::min((size_t)list_cap, cap); ++q) list[k * list_cap + q] = lst[k * cap + q];
  }
  return ABYSS_OK;
}

int irregular_levels(abyss_ac *ac) {
  if (ac->dev_irr) return irregular_levels_device(ac);
  const double t0 = now_s();
#ifdef _OPENMP
  const int nth = std::max(1, omp_get_max_threads());
#else
  const int nth = 1;
#endif
  // the neighbour mirror is refreshed from the particles (the state of record)
  // at every call, and kept current by the commits below
  if ((int)ac->slot.size() != ac->n) build_slots(ac);
#pragma omp parallel for schedule(static) if (ac->n >= 16384)
  for (int i = 0; i < ac->n; ++i) put_rec(ac, i);
  // every particle due before the next regular block, filed under its next
  // irregular level (the order within a level changes nothing, see below)
  std::map<ULL, std::vector<int>> levels;
  if (ac->n >= 16384 && nth > 1) {
    std::vector<std::map<ULL, std::vector<int>>> part(nth);
#pragma omp parallel num_threads(nth)
    {
#ifdef _OPENMP
      std::map<ULL, std::vector<int>> &mine = part[omp_get_thread_num()];
#else
      std::map<ULL, std::vector<int>> &mine = part[0];
#endif
      ULL last = 0;
      std::vector<int> *lv = nullptr;
#pragma omp for schedule(static)
      for (int i = 0; i < ac->n; ++i) {
        const ULL key = ac->s[i].next_irr;
        if (key > ac->next_reg_block) continue;
        if (!lv || key != last) {
          lv = &mine[key];
          last = key;
        }
        lv->push_back(i);
      }
    }
    for (auto &mine : part)
      for (auto &kv : mine) {
        std::vector<int> &dst = levels[kv.first];
        dst.insert(dst.end(), kv.second.begin(), kv.second.end());
      }
  } else {
    for (int i = 0; i < ac->n; ++i)
      if (ac->s[i].next_irr <= ac->next_reg_block) levels[ac->s[i].next_irr].push_back(i);
  }
  std::vector<Filing> filing(nth);
  std::vector<Pending> pend;
  while (!levels.empty()) {
    auto it = levels.begin();
    // The level's particles are computed from the pre-level state and committed
    // one by one, so their order changes nothing.
    std::vector<int> P = std::move(it->second);
    levels.erase(it);
    pend.resize(P.size());
    int bad = 0;
    // small levels, or one thread: no thread team (its set-up costs more than
    // the level)
    if (nth > 1 && P.size() >= 32) {
#pragma omp parallel
      run_level(ac, P, pend, filing, &bad);
    } else {
      run_level(ac, P, pend, filing, &bad);
    }
    if (bad) {
      ac->err = "irregular time step out of range";
      return ABYSS_ERR_STATE;
    }
    for (Filing &f : filing) f.drain_into(levels);
    ac->st.irr_levels++;
    ac->st.irr_steps += (long long)P.size();
  }
  ac->st.sec_irr += now_s() - t0;
  return ABYSS_OK;
}

// Neighbour-change correction of updateRegularParticleCuda
// (ComputeAcceleration.cpp:457-577): walking both lists in step, the force of a
// lost neighbour (old, not new) is subtracted and that of a gained one (new,
// not old) added, in that interleaved order.  pred(j, pos, vel) gives j's
// predicted state.
template <class Pred, class Mass>
void neighbour_change(const int *old_nb, int n_old, const int *new_nb, int n_new, Pred pred,
                      Mass mass, double eps2, const double pos[3], const double vel[3],
                      double a_tmp[3], double adot_tmp[3]) {
  // lost[k]: old_nb[k] is not in the new list; gained[k]: new_nb[k] is not in
  // the old one.  Lists kept by this library are ascending, and a linear merge
  // marks them; other lists go through hash sets.
  thread_local std::vector<char> lost, gained;
  lost.assign(n_old, 0);
  gained.assign(n_new, 0);
  const bool sorted_old = std::is_sorted(old_nb, old_nb + n_old);
  const bool sorted_new = std::is_sorted(new_nb, new_nb + n_new);
  if (sorted_old && sorted_new) {
    int a = 0, b = 0;
    while (a < n_old || b < n_new) {
      if (b >= n_new || (a < n_old && old_nb[a] < new_nb[b])) {
        lost[a++] = 1;
      } else if (a >= n_old || new_nb[b] < old_nb[a]) {
        gained[b++] = 1;
      } else {
        const int v = old_nb[a];  // in both (repeats advance together)
        while (a < n_old && old_nb[a] == v) ++a;
        while (b < n_new && new_nb[b] == v) ++b;
      }
    }
  } else {
    std::unordered_set<int> old_set(old_nb, old_nb + n_old);
    std::unordered_set<int> new_set(new_nb, new_nb + n_new);
    for (int k = 0; k < n_old; ++k) lost[k] = !new_set.count(old_nb[k]);
    for (int k = 0; k < n_new; ++k) gained[k] = !old_set.count(new_nb[k]);
  }
  const int size = std::max(n_old, n_new);
  for (int k = 0; k < size; ++k) {
    if (k < n_old && lost[k]) {
      double pj[3], vj[3];
      pred(old_nb[k], pj, vj);
      pair_force(pos, vel, pj, vj, mass(old_nb[k]), eps2, a_tmp, adot_tmp, -1.0);
    }
    if (k < n_new && gained[k]) {
      double pj[3], vj[3];
      pred(new_nb[k], pj, vj);
      pair_force(pos, vel, pj, vj, mass(new_nb[k]), eps2, a_tmp, adot_tmp, +1.0);
    }
  }
}

// Fourth-order Hermite corrector of a regular step (ComputeAcceleration.cpp:592-632).
void hermite_regular(const double pos[3], const double vel[3], const double a_reg[3][4],
                     const double acc[3], const double jerk[3], const double a_tmp[3],
                     const double adot_tmp[3], double dt, double new_x[3], double new_v[3],
                     double a2o[3], double a3o[3]) {
  const double dt2 = dt * dt, dt3 = dt2 * dt, dt4 = dt3 * dt, dt5 = dt4 * dt;
  for (int d = 0; d < 3; ++d) {
    const double da_dt2 = (a_reg[d][0] - acc[d] - a_tmp[d]) / dt2;
    const double adot_dt = (a_reg[d][1] + jerk[d] + adot_tmp[d]) / dt;
    const double a2 = -6 * da_dt2 - 2 * adot_dt - 2 * a_reg[d][1] / dt;
    const double a3 = (12 * da_dt2 + 6 * adot_dt) / dt;
    new_x[d] = pos[d] + a2 * dt4 / 24 + a3 * dt5 / 120;
    new_v[d] = vel[d] + a2 * dt3 / 6 + a3 * dt4 / 24;
    a2o[d] = a2;
    a3o[d] = a3;
  }
}

// Assemble the new regular/irregular/total derivatives (ComputeAcceleration.cpp:647-660).
void commit_derivatives(const double acc[3], const double jerk[3], const double airr[3],
                        const double jirr[3], const double a2[3], const double a3[3], int nnb,
                        double a_reg[3][4], double a_irr[3][4], double a_tot[3][4]) {
  for (int d = 0; d < 3; ++d) {
    a_reg[d][2] = a2[d];
    a_reg[d][3] = a3[d];
    a_reg[d][0] = acc[d];
    a_reg[d][1] = jerk[d];
    a_irr[d][0] = airr[d];
    a_irr[d][1] = jirr[d];
    a_tot[d][0] = a_reg[d][0] + a_irr[d][0];
    a_tot[d][1] = a_reg[d][1] + a_irr[d][1];
    if (nnb == 0) {
      a_tot[d][2] = a_reg[d][2];
      a_tot[d][3] = a_reg[d][3];
    }
  }
}

// updateRegularParticleCuda (ComputeAcceleration.cpp:405-661) for one target
// of a regular call, with the irregular part taken from the device (FP64 over
// the new list, same predicted positions).
void regular_correct_one(const abyss_ac *ac, int i, const double *acc, const double *jerk,
                         const double *airr, const double *jirr, const int *lst, int nnb,
                         Pending &out) {
  const Star &p = ac->s[i];
  const double new_time = p.t_reg + p.dt_reg;
  double pos[3], vel[3];
  predict(p, p.nb.empty() ? p.dt_reg : 0.0, ac->scale, pos, vel);
  double a_tmp[3] = {0, 0, 0}, adot_tmp[3] = {0, 0, 0};
  auto pred = [&](int j, double pj[3], double vj[3]) {
    const Star &q = ac->s[j];
    predict(q, new_time - (q.nb.empty() ? q.t_reg : q.t_irr), ac->scale, pj, vj);
  };
  auto mass = [&](int j) { return ac->s[j].m; };
  neighbour_change(p.nb.data(), (int)p.nb.size(), lst, nnb, pred, mass, ac->p.eps2, pos, vel, a_tmp,
                   adot_tmp);
  const double dt = p.dt_reg * ac->scale;
  double a2[3], a3[3];
  hermite_regular(pos, vel, p.a_reg, acc, jerk, a_tmp, adot_tmp, dt, out.new_x, out.new_v, a2, a3);
  std::memcpy(out.a_reg, p.a_reg, sizeof(out.a_reg));
  std::memcpy(out.a_irr, p.a_irr, sizeof(out.a_irr));
  std::memcpy(out.a_tot, p.a_tot, sizeof(out.a_tot));
  commit_derivatives(acc, jerk, airr, jirr, a2, a3, nnb, out.a_reg, out.a_irr, out.a_tot);
  out.new_nb.assign(lst, lst + nnb);
  out.move = true;
}

// The host half of a regular block once the force is known: corrector and
// commit for every target (results in target order, lists [m][cap]).  The
// result vectors are kept, moved, as the last call's record.
int finish_regular(abyss_ac *ac, const std::vector<int> &targets, std::vector<double> &&acc,
                   std::vector<double> &&jerk, const std::vector<double> &airr, const std::vector<double> &jirr,
                   std::vector<int> &&nnb, std::vector<int> &&lst, int cap);

int regular_block(abyss_ac *ac, const std::vector<int> &targets) {
  const double new_time = ac->next_reg_block * ac->time_step;
  // the last block's result buffers are reused (finish_regular moves this
  // block's back into the record), so that no block allocates or clears them
  std::vector<double> acc = std::move(ac->last_acc), jerk = std::move(ac->last_jerk), airr, jirr;
  std::vector<int> nnb = std::move(ac->last_nnb), lst = std::move(ac->last_list);
  ac->last_targets.clear();  // no record until this block's is complete
  airr.swap(ac->reg_airr);
  jirr.swap(ac->reg_jirr);
  struct Back {  // the FP64 irregular parts' buffers go back too
    abyss_ac *ac;
    std::vector<double> &a, &j;
    ~Back() {
      ac->reg_airr.swap(a);
      ac->reg_jirr.swap(j);
    }
  } back{ac, airr, jirr};
  for (int attempt = 0;; ++attempt) {
    int rc = upload_and_predict(ac, new_time);
    if (rc != ABYSS_OK) return rc;
    rc = regular_gpu(ac, targets, true, acc, jerk, airr, jirr, nnb, lst);
    if (rc == ABYSS_OK) break;
    if (rc != 2 || attempt > 40) return rc < 0 ? rc : ABYSS_ERR_STATE;
  }
  return finish_regular(ac, targets, std::move(acc), std::move(jerk), airr, jirr, std::move(nnb), std::move(lst),
                        ac->p.nb_max);
}

int finish_regular(abyss_ac *ac, const std::vector<int> &targets, std::vector<double> &&acc,
                   std::vector<double> &&jerk, const std::vector<double> &airr, const std::vector<double> &jirr,
                   std::vector<int> &&nnb, std::vector<int> &&lst, int cap) {
  const int m = (int)targets.size();
  const double t0 = now_s();
  std::vector<Pending> pend(m);
  // an exception cannot leave an OpenMP loop: a failed allocation is counted
  // and reported after it, before anything is committed
  int failed = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : failed)
  for (int k = 0; k < m; ++k) {
    try {
      regular_correct_one(ac, targets[k], &acc[3 * (size_t)k], &jerk[3 * (size_t)k], &airr[3 * (size_t)k],
                          &jirr[3 * (size_t)k], &lst[(size_t)k * cap], nnb[k], pend[k]);
    } catch (const std::bad_alloc &) {
      failed++;
    }
  }
  if (failed) {
    ac->err = "regular block: host allocation failed";
    return ABYSS_ERR_OOM;
  }
  // the last call's record (abyss_ac_last_regular) is copied before the commit,
  // so that nothing after the first committed particle allocates; so is the
  // device irregular phase's list of particles to send up again
  ac->last_targets = targets;
  if (ac->dev_irr) ac->eng_dirty.insert(ac->eng_dirty.end(), targets.begin(), targets.end());
  ac->st.pairs += (double)m * ac->n;
  // RegCudaUpdate (WorkerRoutines.cpp:124-143), committed after every corrector ran
  int bad = 0;
  for (int k = 0; k < m; ++k) {
    Star &p = ac->s[targets[k]];
    Pending &q = pend[k];
    p.nb = std::move(q.new_nb);
    std::memcpy(p.a_reg, q.a_reg, sizeof(p.a_reg));
    std::memcpy(p.a_irr, q.a_irr, sizeof(p.a_irr));
    std::memcpy(p.a_tot, q.a_tot, sizeof(p.a_tot));
    for (int d = 0; d < 3; ++d) {
      p.x[d] = q.new_x[d];
      p.v[d] = q.new_v[d];
    }
  }
#pragma omp parallel for schedule(static) reduction(+ : bad)
  for (int k = 0; k < m; ++k) {
    Star &p = ac->s[targets[k]];
    p.cur_reg = p.cur_reg + p.tb_reg;
    p.t_reg = p.cur_reg * ac->time_step;
    try {
      time_step_reg(ac, p);
      time_step_irr(ac, p);
    } catch (const std::exception &) {
      bad++;
    }
    if (p.nb.empty()) {
      p.cur_irr = p.cur_reg;
      p.t_irr = p.cur_reg * ac->time_step;
    }
    update_radius(ac, p);
    p.next_irr = p.cur_irr + p.tb_irr;
  }
  // the last call, for parity checks (abyss_ac_last_regular)
  ac->last_acc = std::move(acc);
  ac->last_jerk = std::move(jerk);
  ac->last_nnb = std::move(nnb);
  ac->last_list = std::move(lst);
  ac->last_cap = cap;
  ac->st.sec_reg_host += now_s() - t0;
  if (bad) {
    ac->err = "regular time step out of range";
    return ABYSS_ERR_STATE;
  }
  ac->st.reg_steps += m;
  ac->st.blocks++;
  return ABYSS_OK;
}

}  // namespace

extern "C" {

int abyss_ac_create(abyss_ctx *ctx, const abyss_ac_params *p, int n, const double *x, const double *v,
                    const double *mass, const double *r2nb, abyss_ac **out) {
  if (!ctx || !p || n < 2 || !x || !v || !mass || !r2nb || !out) return ABYSS_ERR_ARG;
  if (p->nb_max <= 0 || p->fix_nb <= 0 || p->fix_nb >= p->nb_max || !(p->t_end > 0) ||
      !(p->eta_reg > 0) || !(p->eta_irr > 0) || !(p->eps2 >= 0))
    return ABYSS_ERR_ARG;
  abyss_ac *ac = new abyss_ac;
  ac->ctx = ctx;
  ac->p = *p;
  ac->n = n;
  ac->scale = p->t_end;
  ac->s.resize(n);
  for (int i = 0; i < n; ++i) {
    Star &s = ac->s[i];
    for (int d = 0; d < 3; ++d) {
      s.x[d] = x[3 * (size_t)i + d];
      s.v[d] = v[3 * (size_t)i + d];
    }
    s.m = mass[i];
  }
  int rc;
  try {
    rc = initialise(ac, r2nb);
  } catch (const std::exception &e) {
    ac->err = e.what();
    rc = ABYSS_ERR_STATE;
  }
  if (rc != ABYSS_OK) {
    delete ac;
    return rc;
  }
  *out = ac;
  return ABYSS_OK;
}

namespace {

// Shared state of one abyss_ac_serve_run call.
struct ServeRun {
  abyss_ens *e = nullptr;
  abyss_ac *const *acs = nullptr;
  const int *slots = nullptr;
  int k = 0, cap = 0;
  std::mutex mu;
  std::condition_variable cv_host, cv_gpu;
  std::deque<int> host_q;         // integrations with host work to do
  std::vector<int> gpu_ready;     // integrations whose open block is staged
  std::vector<char> has_result;   // a wave result waits for end_block
  std::vector<std::vector<double>> res_d;  // acc, jerk, acc_irr, jerk_irr [4][3m]
  std::vector<std::vector<int>> res_n, res_l;
  int busy = 0;                   // workers inside an integration
  double worker_s = 0.0;          // busy time summed over workers
  int finished = 0;               // integrations that reached code time 1
  bool stop = false, quit = false;
  int *status = nullptr, *blocks = nullptr;
};

// One host worker: takes an integration, commits its returned block if it has
// one, then (unless stopping) opens its next block and stages it for the GPU.
void serve_worker(ServeRun *R) {
  for (;;) {
    int i;
    {
      std::unique_lock<std::mutex> lk(R->mu);
      R->cv_host.wait(lk, [&] { return R->quit || !R->host_q.empty(); });
      if (R->host_q.empty()) return;
      i = R->host_q.front();
      R->host_q.pop_front();
      ++R->busy;
    }
    const double tw = now_s();
    abyss_ac *ac = R->acs[i];
    int st = R->status[i];
    bool queue_gpu = false, fin = false;
    if (R->has_result[i]) {
      const auto &d = R->res_d[i];
      const size_t m3 = d.size() / 4;
      int done = 0;
      const int r = abyss_ac_end_block(ac, d.data(), d.data() + m3, d.data() + 2 * m3, d.data() + 3 * m3,
                                       R->res_n[i].data(), R->res_l[i].data(), R->cap, &done);
      R->has_result[i] = 0;
      if (r == ABYSS_WARN_OVERFLOW) {
        st = ABYSS_ROUND_REDO;
      } else if (r != ABYSS_OK) {
        st = r;
      } else {
        ++R->blocks[i];
        st = done ? ABYSS_ROUND_ADVANCED_DONE : ABYSS_ROUND_ADVANCED;
        fin = done != 0;
      }
    }
    bool stopping;
    {
      std::lock_guard<std::mutex> lk(R->mu);
      stopping = R->stop;
    }
    if (st >= 0 && !fin && !stopping) {
      if (!ac->in_block) {
        int m = 0, done = 0;
        double nt = 0.0, sc = 1.0;
        const int r = abyss_ac_begin_block(ac, &m, &nt, &sc, &done);
        if (r != ABYSS_OK) {
          st = r;
        } else if (done || m == 0) {
          st = ABYSS_ROUND_FINISHED;
          fin = true;
        }
      }
      if (st >= 0 && !fin) {
        double *x, *v, *a0, *a1, *t0, *ms, *r2;
        int r = abyss_ens_stage(R->e, R->slots[i], &x, &v, &a0, &a1, &t0, &ms, &r2);
        if (r == ABYSS_OK) r = abyss_ac_block_state(ac, x, v, a0, a1, t0, ms, r2);
        if (r != ABYSS_OK)
          st = r;
        else
          queue_gpu = true;
      }
    }
    {
      std::lock_guard<std::mutex> lk(R->mu);
      R->status[i] = st;
      if (fin) ++R->finished;
      if (queue_gpu) R->gpu_ready.push_back(i);
      --R->busy;
      R->worker_s += now_s() - tw;
    }
    R->cv_gpu.notify_one();
  }
}

}  // namespace

int abyss_ac_serve_run(abyss_ens *e, int k, abyss_ac *const *acs, const int *slots, double eps2, int mode,
                       int threads, double budget_ms, int stop_after, int *status, int *blocks, float *gpu_ms,
                       int *waves, abyss_serve_stats *stats) {
  if (!e || k < 0 || (k > 0 && (!acs || !slots || !status || !blocks))) return ABYSS_ERR_ARG;
  if (gpu_ms) *gpu_ms = 0.0f;
  if (waves) *waves = 0;
  if (k == 0) return ABYSS_OK;
  for (int i = 0; i < k; ++i)
    if (!acs[i]) return ABYSS_ERR_ARG;
  int rc = abyss_ens_stage_reserve(e);
  if (rc != ABYSS_OK) return rc;
  ServeRun R;
  R.e = e;
  R.acs = acs;
  R.slots = slots;
  R.k = k;
  R.cap = abyss_ens_list_cap(e);
  R.status = status;
  R.blocks = blocks;
  R.has_result.assign(k, 0);
  R.res_d.resize(k);
  R.res_n.resize(k);
  R.res_l.resize(k);
  for (int i = 0; i < k; ++i) {
    status[i] = ABYSS_ROUND_ADVANCED;
    blocks[i] = 0;
    R.host_q.push_back(i);
  }
  const int nth = std::max(1, threads > 0 ? threads : (int)std::thread::hardware_concurrency());
  std::vector<std::thread> pool;
  for (int t = 0; t < nth; ++t) pool.emplace_back(serve_worker, &R);
  const double t0 = now_s();
  const int want_fin = stop_after > 0 ? std::min(stop_after, k) : k;
  int err = ABYSS_OK;
  abyss_serve_stats S{};
  // The dispatcher: every staged block goes into the next wave.  Two waves can
  // be in flight: while the GPU runs one, the next is uploaded and launched
  // behind it, or the last one's rows are handed back.
  struct Flight {
    int ticket;
    std::vector<int> wave, mper;
  };
  std::deque<Flight> infl;
  for (;;) {
    std::vector<int> wave;
    bool collect = false;
    double tp = now_s();
    {
      std::unique_lock<std::mutex> lk(R.mu);
      for (;;) {
        if (!R.gpu_ready.empty() && infl.size() < 2) {
          wave.swap(R.gpu_ready);
          break;
        }
        if (!infl.empty()) {
          lk.unlock();
          const int r = abyss_ens_ready(e, infl.front().ticket);
          lk.lock();
          if (r != 0) {  // finished (or failed: collect reports it)
            collect = true;
            break;
          }
          R.cv_gpu.wait_for(lk, std::chrono::microseconds(20));
          continue;
        }
        if (R.busy == 0 && R.host_q.empty()) break;  // all done or stopped
        R.cv_gpu.wait(lk);
      }
    }
    S.idle_s += now_s() - tp;
    if (wave.empty() && !collect) break;
    tp = now_s();
    if (!wave.empty()) {
      std::vector<int> cl, mper, tg;
      std::vector<double> tm, scl;
      for (int i : wave) {
        const abyss_ac *ac = acs[i];
        cl.push_back(slots[i]);
        tm.push_back(ac->next_reg_block * ac->time_step);
        scl.push_back(ac->scale);
        mper.push_back((int)ac->block_targets.size());
        tg.insert(tg.end(), ac->block_targets.begin(), ac->block_targets.end());
      }
      int ticket = -1;
      rc = abyss_ens_submit(e, (int)wave.size(), cl.data(), tm.data(), scl.data(), mper.data(), tg.data(), eps2,
                            mode, &ticket);
      S.prep_s += now_s() - tp;
      if (rc != ABYSS_OK) {
        err = rc;
        break;
      }
      S.rows += (long long)tg.size();
      infl.push_back(Flight{ticket, std::move(wave), std::move(mper)});
      continue;
    }
    // hand the oldest wave's rows back to the workers
    Flight f = std::move(infl.front());
    infl.pop_front();
    const double *acc, *jerk, *airr, *jirr;
    const int *nnb, *lst;
    int rows = 0;
    float ms = 0.0f;
    rc = abyss_ens_collect(e, f.ticket, &acc, &jerk, &airr, &jirr, &nnb, &lst, &rows, &ms);
    if (rc == ABYSS_WARN_OVERFLOW) rc = ABYSS_OK;  // end_block handles each overflowed block
    S.wait_s += now_s() - tp;
    if (rc != ABYSS_OK) {
      err = rc;
      break;
    }
    tp = now_s();
    if (gpu_ms) *gpu_ms += ms;
    if (waves) ++*waves;
    // the wave's integrations are idle until their rows are handed back, so
    // their result buffers are filled without the lock
    size_t r0 = 0;
    for (size_t b = 0; b < f.wave.size(); ++b) {
      const int i = f.wave[b];
      const size_t m = f.mper[b];
      auto &d = R.res_d[i];
      d.resize(12 * m);
      std::copy(acc + 3 * r0, acc + 3 * (r0 + m), d.begin());
      std::copy(jerk + 3 * r0, jerk + 3 * (r0 + m), d.begin() + 3 * m);
      std::copy(airr + 3 * r0, airr + 3 * (r0 + m), d.begin() + 6 * m);
      std::copy(jirr + 3 * r0, jirr + 3 * (r0 + m), d.begin() + 9 * m);
      R.res_n[i].assign(nnb + r0, nnb + r0 + m);
      R.res_l[i].assign(lst + r0 * R.cap, lst + (r0 + m) * R.cap);
      R.has_result[i] = 1;
      r0 += m;
    }
    {
      std::lock_guard<std::mutex> lk(R.mu);
      for (int i : f.wave) R.host_q.push_back(i);
      if (R.finished >= want_fin || (budget_ms > 0 && (now_s() - t0) * 1e3 >= budget_ms)) R.stop = true;
    }
    R.cv_host.notify_all();
    S.hand_s += now_s() - tp;
  }
  if (err != ABYSS_OK) {
    // drain what is in flight so that the ensemble is usable again
    for (const Flight &f : infl) {
      const double *a, *b2, *c2, *d2;
      const int *n2, *l2;
      int rows = 0;
      (void)abyss_ens_collect(e, f.ticket, &a, &b2, &c2, &d2, &n2, &l2, &rows, nullptr);
    }
    std::lock_guard<std::mutex> lk(R.mu);
    R.stop = true;
    R.host_q.clear();
  }
  {
    std::lock_guard<std::mutex> lk(R.mu);
    R.quit = true;
  }
  R.cv_host.notify_all();
  for (auto &t : pool) t.join();
  if (stats) {
    S.wall_s = now_s() - t0;
    S.worker_s = R.worker_s;
    *stats = S;
  }
  return err;
}

int abyss_ac_destroy(abyss_ac *ac) {
  delete ac;
  return ABYSS_OK;
}

int abyss_ac_host_timers(const abyss_ac *ac, double *sec2) {
  if (!ac || !sec2) return ABYSS_ERR_ARG;
  sec2[0] = ac->sec_jset;
  sec2[1] = ac->sec_sched;
  return ABYSS_OK;
}

int abyss_ac_set_device_irregular(abyss_ac *ac, int on) {
  if (!ac) return ABYSS_ERR_ARG;
  if (ac->in_block) {
    ac->err = "set_device_irregular: a split block is open";
    return ABYSS_ERR_STATE;
  }
  if (on && !ac->ctx) {
    ac->err = "set_device_irregular: the integration has no GPU context";
    return ABYSS_ERR_STATE;
  }
  if (ac->dev_res) {  // the device's copy stays the state of record
    ac->dev_irr = on != 0;
    return ABYSS_OK;
  }
  ac->dev_irr = on != 0;
  ac->eng_synced = false;  // the host may have stepped particles meanwhile
  ac->eng_dirty.clear();
  return ABYSS_OK;
}

int abyss_ac_set_device_resident(abyss_ac *ac, int on) {
  if (!ac) return ABYSS_ERR_ARG;
  if (ac->in_block) {
    ac->err = "set_device_resident: a split block is open";
    return ABYSS_ERR_STATE;
  }
  if (on && !ac->ctx) {
    ac->err = "set_device_resident: the integration has no GPU context";
    return ABYSS_ERR_STATE;
  }
  if ((on != 0) == ac->dev_res) return ABYSS_OK;
  if (on) {
    ac->eng_synced = false;  // the first device block sends every particle up
    ac->host_stale = false;
    ac->res_last_m = 0;
    ac->dev_res = true;
    return ABYSS_OK;
  }
  const int rc = resident_sync_host(ac);
  if (rc != ABYSS_OK) return rc;
  ac->dev_res = false;
  ac->eng_synced = false;  // a later device irregular phase sends every particle up
  ac->eng_dirty.clear();
  // the host's last-call record is of a block before the switch
  ac->last_targets.clear();
  return ABYSS_OK;
}

int abyss_ac_device_resident_info(const abyss_ac *ac, int *on, long long *borderline, double *sec_sync) {
  if (!ac) return ABYSS_ERR_ARG;
  if (on) *on = ac->dev_res ? 1 : 0;
  if (borderline) *borderline = ac->res_borderline;
  if (sec_sync) *sec_sync = ac->res_sec_sync;
  return ABYSS_OK;
}

int abyss_ac_device_irregular_info(const abyss_ac *ac, int *on, long long *borderline, double *sec_copy,
                                   long long *cycles6) {
  if (!ac) return ABYSS_ERR_ARG;
  if (on) *on = ac->dev_irr ? 1 : 0;
  if (cycles6)
    for (int q = 0; q < 6; ++q) cycles6[q] = ac->dev_cycles[q];
  if (borderline) *borderline = ac->dev_borderline;
  if (sec_copy) *sec_copy = ac->dev_sec_copy;
  return ABYSS_OK;
}

int abyss_device_irregular_steps(int device, int n, const double *x, const double *v, const double *mass,
                                 const double *a_tot, const double *a_reg, const double *a_irr,
                                 const double *t_reg, const double *t_irr, const double *dt_irr,
                                 const int *nnb, const int *nb, int nb_stride, double eps2, double scale,
                                 int time_block, double eta_irr, const int *lv_reg,
                                 const unsigned long long *cur_reg, const unsigned long long *tb_reg, int count,
                                 const int *idx, double *new_pos, double *new_vel, double *a_irr_out,
                                 double *a_tot_out, int *lv_irr_out, double *dt_irr_out,
                                 unsigned long long *tb_irr_out) {
  if (n <= 0 || count < 0 || nb_stride <= 0 || !x || !v || !mass || !a_tot || !a_reg || !a_irr || !t_reg ||
      !t_irr || !dt_irr || !nnb || !lv_reg || !cur_reg || !tb_reg || time_block < -62 || time_block > -1 ||
      (count > 0 && (!idx || !new_pos || !new_vel || !a_irr_out || !a_tot_out)))
    return ABYSS_ERR_ARG;
  for (int i = 0; i < n; ++i) {
    if (nnb[i] < 0 || nnb[i] > nb_stride || (nnb[i] > 0 && !nb)) return ABYSS_ERR_ARG;
    for (int k = 0; k < nnb[i]; ++k) {
      const int j = nb[(size_t)i * nb_stride + k];
      if (j < 0 || j >= n || j == i) return ABYSS_ERR_ARG;
    }
  }
  for (int k = 0; k < count; ++k)
    if (idx[k] < 0 || idx[k] >= n) return ABYSS_ERR_ARG;
  using namespace abyss_irr;
  Engine *e = nullptr;
  int rc = engine_create(device, &e);
  if (rc != ABYSS_OK) return rc;
  std::unique_ptr<Engine, void (*)(Engine *)> hold(e, engine_destroy);
  if ((rc = engine_reserve(e, n, nb_stride)) != ABYSS_OK) return rc;
  Image *img = engine_images(e);
  int *lists = engine_lists(e);
  const double step = pow2(time_block);
  for (int i = 0; i < n; ++i) {
    Image &g = img[i];
    for (int d = 0; d < 3; ++d) {
      g.x[d] = x[3 * (size_t)i + d];
      g.v[d] = v[3 * (size_t)i + d];
    }
    g.m = mass[i];
    g.t_irr = t_irr[i];
    g.t_reg = t_reg[i];
    g.dt_irr = dt_irr[i];
    std::memcpy(g.a_tot, a_tot + 12 * (size_t)i, sizeof(g.a_tot));
    std::memcpy(g.a_reg, a_reg + 12 * (size_t)i, sizeof(g.a_reg));
    std::memcpy(g.a_irr, a_irr + 12 * (size_t)i, sizeof(g.a_irr));
    // block counts of times on the 2^time_block grid, the level of the step
    g.cur_irr = (ULL)(t_irr[i] / step);
    g.tb_irr = (ULL)(dt_irr[i] / step);
    g.next_irr = g.cur_irr + g.tb_irr;
    g.new_cur_irr = 0;
    g.cur_reg = cur_reg[i];
    g.tb_reg = tb_reg[i];
    g.lv_irr = dt_irr[i] > 0 ? std::ilogb(dt_irr[i]) : time_block;
    g.lv_reg = lv_reg[i];
    g.nnb = nnb[i];
    g.index = i;
    g.list_off = (long long)i * nb_stride;
    if (nnb[i] > 0) std::memcpy(lists + (size_t)i * nb_stride, nb + (size_t)i * nb_stride, sizeof(int) * nnb[i]);
  }
  if ((rc = engine_upload(e, n, (long long)n * nb_stride)) != ABYSS_OK) return rc;
  Params P;
  P.scale = scale;
  P.time_step = step;
  P.eps2 = eps2;
  P.eta_irr = eta_irr;
  P.ln2 = std::log(2.0);
  P.time_block = time_block;
  P.next_reg_block = 0;
  return engine_steps(e, P, count, idx, new_pos, new_vel, a_irr_out, a_tot_out, lv_irr_out, dt_irr_out, tb_irr_out);
}

namespace {
// updateNextRegTime (RootRoutines.cpp:1310-1338): the next regular block time
// and its particles, in ascending index.
std::vector<int> next_regular_block(abyss_ac *ac) {
  struct Clock {
    abyss_ac *ac;
    double t0 = now_s();
    ~Clock() { ac->sec_sched += now_s() - t0; }
  } clock{ac};
  ULL tmin = ac->block_max;
  std::vector<int> targets;
  for (int i = 0; i < ac->n; ++i) {
    const ULL t = ac->s[i].cur_reg + ac->s[i].tb_reg;
    if (t <= tmin) {
      if (t < tmin) {
        targets.clear();
        tmin = t;
      }
      targets.push_back(i);
    }
  }
  ac->next_reg_block = tmin;
  return targets;
}
}  // namespace

int abyss_ac_advance_block(abyss_ac *ac, int *done) {
  if (!ac) return ABYSS_ERR_ARG;
  if (ac->in_block) {
    ac->err = "advance_block: a split block is open";
    return ABYSS_ERR_STATE;
  }
  set_threads(ac);
  if (ac->done || ac->next_reg_block * ac->time_step >= 1) {
    ac->done = true;
    if (done) *done = 1;
    return ABYSS_OK;
  }
  if (ac->dev_res) {
    const int rc = resident_block(ac);
    if (rc != ABYSS_OK) return rc;
    if (ac->next_reg_block * ac->time_step >= 1) ac->done = true;
    if (done) *done = ac->done ? 1 : 0;
    return ABYSS_OK;
  }
  std::vector<int> targets = next_regular_block(ac);
  int rc = irregular_levels(ac);
  if (rc != ABYSS_OK) return rc;
  try {
    rc = regular_block(ac, targets);
  } catch (const std::exception &e) {
    ac->err = e.what();
    rc = ABYSS_ERR_STATE;
  }
  if (rc != ABYSS_OK) return rc;
  if (ac->next_reg_block * ac->time_step >= 1) ac->done = true;
  if (done) *done = ac->done ? 1 : 0;
  return ABYSS_OK;
}

int abyss_ac_begin_block(abyss_ac *ac, int *m, double *new_time, double *time_scale, int *done) {
  if (!ac || !m) return ABYSS_ERR_ARG;
  if (ac->in_block) {
    ac->err = "begin_block: a block is already open";
    return ABYSS_ERR_STATE;
  }
  if (ac->dev_res) {
    ac->err = "begin_block: the state is resident on the device (abyss_ac_set_device_resident)";
    return ABYSS_ERR_STATE;
  }
  set_threads(ac);
  if (ac->done || ac->next_reg_block * ac->time_step >= 1) {
    ac->done = true;
    *m = 0;
    if (done) *done = 1;
    return ABYSS_OK;
  }
  ac->block_targets = next_regular_block(ac);
  int rc;
  try {
    rc = irregular_levels(ac);
  } catch (const std::exception &e) {
    ac->err = e.what();
    rc = ABYSS_ERR_STATE;
  }
  if (rc != ABYSS_OK) return rc;
  ac->in_block = true;
  *m = (int)ac->block_targets.size();
  if (new_time) *new_time = ac->next_reg_block * ac->time_step;
  if (time_scale) *time_scale = ac->scale;
  if (done) *done = 0;
  return ABYSS_OK;
}

int abyss_ac_block_targets(const abyss_ac *ac, int *targets) {
  if (!ac || !targets || !ac->in_block) return ABYSS_ERR_ARG;
  std::copy(ac->block_targets.begin(), ac->block_targets.end(), targets);
  return ABYSS_OK;
}

int abyss_ac_block_state(const abyss_ac *ac, double *x, double *v, double *a0, double *a1, double *t0,
                         double *mass, double *r2nb) {
  if (!ac || !x || !v || !a0 || !a1 || !t0 || !mass || !r2nb) return ABYSS_ERR_ARG;
  for (int j = 0; j < ac->n; ++j) {
    const Star &p = ac->s[j];
    for (int d = 0; d < 3; ++d) {
      x[3 * (size_t)j + d] = p.x[d];
      v[3 * (size_t)j + d] = p.v[d];
      a0[3 * (size_t)j + d] = p.a_tot[d][0];
      a1[3 * (size_t)j + d] = p.a_tot[d][1];
    }
    t0[j] = p.nb.empty() ? p.t_reg : p.t_irr;  // CalculateRegularAcceleration.cpp:371-374
    mass[j] = p.m;
    r2nb[j] = p.r2nb;
  }
  return ABYSS_OK;
}

int abyss_ac_end_block(abyss_ac *ac, const double *acc, const double *jerk, const double *acc_irr,
                       const double *jerk_irr, const int *nnb, const int *list, int list_cap, int *done) {
  if (!ac || !acc || !jerk || !acc_irr || !jerk_irr || !nnb || !list || list_cap <= 0) return ABYSS_ERR_ARG;
  if (!ac->in_block) {
    ac->err = "end_block: no block is open";
    return ABYSS_ERR_STATE;
  }
  set_threads(ac);
  const int m = (int)ac->block_targets.size();
  // results from the caller are checked before anything is used: a negative
  // count or a neighbour index outside the cluster is refused, block left open
  for (int k = 0; k < m; ++k) {
    if (nnb[k] < 0) {
      ac->err = "end_block: negative neighbour count in row " + std::to_string(k);
      return ABYSS_ERR_ARG;
    }
    const int q = nnb[k] < list_cap ? nnb[k] : list_cap;
    const int *row = list + (size_t)k * list_cap;
    for (int i = 0; i < q; ++i)
      if (row[i] < 0 || row[i] >= ac->n) {
        ac->err = "end_block: neighbour index " + std::to_string(row[i]) + " outside the cluster in row " +
                  std::to_string(k);
        return ABYSS_ERR_ARG;
      }
  }
  // a list that did not fit: shrink those radii, commit nothing, ask for a redo
  bool over = false;
  for (int k = 0; k < m; ++k)
    if (nnb[k] > list_cap) {
      ac->s[ac->block_targets[k]].r2nb *= 0.8;
      over = true;
    }
  if (over) {
    ac->st.radius_retries++;
    return ABYSS_WARN_OVERFLOW;
  }
  int rc;
  try {
    std::vector<double> va(acc, acc + 3 * (size_t)m), vj(jerk, jerk + 3 * (size_t)m),
        vai(acc_irr, acc_irr + 3 * (size_t)m), vji(jerk_irr, jerk_irr + 3 * (size_t)m);
    std::vector<int> vn(nnb, nnb + m), vl(list, list + (size_t)m * list_cap);
    rc = finish_regular(ac, ac->block_targets, std::move(va), std::move(vj), vai, vji, std::move(vn), std::move(vl),
                        list_cap);
  } catch (const std::bad_alloc &) {
    ac->err = "end_block: host allocation failed";
    rc = ABYSS_ERR_OOM;
  } catch (const std::exception &e) {
    ac->err = e.what();
    rc = ABYSS_ERR_STATE;
  }
  // an allocation failure happens before the commit: the block stays open and
  // end_block may be called again
  if (rc != ABYSS_ERR_OOM) ac->in_block = false;
  if (rc != ABYSS_OK) return rc;
  if (ac->next_reg_block * ac->time_step >= 1) ac->done = true;
  if (done) *done = ac->done ? 1 : 0;
  return ABYSS_OK;
}

int abyss_ac_run(abyss_ac *ac, double t_code) {
  if (!ac) return ABYSS_ERR_ARG;
  int done = 0;
  while (!done && ac->next_reg_block * ac->time_step < t_code) {
    int rc = abyss_ac_advance_block(ac, &done);
    if (rc != ABYSS_OK) return rc;
  }
  return ABYSS_OK;
}

double abyss_ac_time(const abyss_ac *ac) { return ac ? ac->next_reg_block * ac->time_step : 0.0; }

int abyss_ac_get_state(const abyss_ac *ac, double *x, double *v, int *nnb, double *r2nb) {
  if (!ac) return ABYSS_ERR_ARG;
  const int rc = resident_sync_host(ac);
  if (rc != ABYSS_OK) return rc;
  for (int i = 0; i < ac->n; ++i) {
    const Star &s = ac->s[i];
    for (int d = 0; d < 3; ++d) {
      if (x) x[3 * (size_t)i + d] = s.x[d];
      if (v) v[3 * (size_t)i + d] = s.v[d];
    }
    if (nnb) nnb[i] = (int)s.nb.size();
    if (r2nb) r2nb[i] = s.r2nb;
  }
  return ABYSS_OK;
}

int abyss_ac_energy(abyss_ac *ac, double *energy) {
  if (!ac || !energy) return ABYSS_ERR_ARG;
  std::vector<double> x(3 * (size_t)ac->n), v(3 * (size_t)ac->n), m(ac->n);
  int rc = abyss_ac_get_state(ac, x.data(), v.data(), nullptr, nullptr);
  if (rc != ABYSS_OK) return rc;
  for (int i = 0; i < ac->n; ++i) m[i] = ac->s[i].m;
  rc = abyss_energy(ac->ctx, ac->n, x.data(), v.data(), m.data(), ac->p.eps2, energy);
  if (rc != ABYSS_OK) ac->err = abyss_last_error(ac->ctx);
  return rc;
}

int abyss_ac_get_stats(const abyss_ac *ac, abyss_ac_stats *st) {
  if (!ac || !st) return ABYSS_ERR_ARG;
  *st = ac->st;
  return ABYSS_OK;
}

int abyss_ac_last_regular(const abyss_ac *ac, int *m, int *targets, double *px, double *pv,
                          double *r2nb, double *acc_reg, double *jerk_reg, int *nnb, int *list,
                          int list_cap) {
  if (!ac || !m) return ABYSS_ERR_ARG;
  if (ac->dev_res) return resident_last_regular(ac, m, targets, px, pv, r2nb, acc_reg, jerk_reg, nnb, list, list_cap);
  const int mm = (int)ac->last_targets.size();
  const size_t M = mm;
  if (ac->last_acc.size() < 3 * M || ac->last_jerk.size() < 3 * M || ac->last_nnb.size() < M ||
      ac->last_list.size() < M * (size_t)ac->last_cap) {
    *m = 0;
    return ABYSS_ERR_STATE;  // a block failed after taking the record's buffers
  }
  *m = mm;
  if (px || pv) {
    int rc = abyss_read_predicted(ac->ctx, px, pv, nullptr);
    if (rc != ABYSS_OK) return rc;
  }
  for (int k = 0; k < mm; ++k) {
    if (targets) targets[k] = ac->last_targets[k];
    for (int d = 0; d < 3; ++d) {
      if (acc_reg) acc_reg[3 * (size_t)k + d] = ac->last_acc[3 * (size_t)k + d];
      if (jerk_reg) jerk_reg[3 * (size_t)k + d] = ac->last_jerk[3 * (size_t)k + d];
    }
    if (nnb) nnb[k] = ac->last_nnb[k];
    if (list)
      for (int q = 0; q < std::min(list_cap, ac->last_cap); ++q)
        list[(size_t)k * list_cap + q] = ac->last_list[(size_t)k * ac->last_cap + q];
  }
  if (r2nb)
    for (size_t j = 0; j < ac->last_r2.size(); ++j) r2nb[j] = ac->last_r2[j];
  return ABYSS_OK;
}

const char *abyss_ac_last_error(const abyss_ac *ac) { return ac ? ac->err.c_str() : "null integrator"; }

int abyss_ac_info(const abyss_ac *ac, int *n, abyss_ac_params *p) {
  if (!ac) return ABYSS_ERR_ARG;
  if (n) *n = ac->n;
  if (p) *p = ac->p;
  return ABYSS_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ host rules
// The integrator's per-particle rules, exported so they can be checked against
// the reference's outputs without a GPU (include/abyss_host.h).
extern "C" {

void abyss_host_predict(const double *x, const double *v, const double *a0, const double *a1,
                        double dt_code, double scale, double *pos, double *vel) {
  Star p{};
  for (int d = 0; d < 3; ++d) {
    p.x[d] = x[d];
    p.v[d] = v[d];
    p.a_tot[d][0] = a0[d];
    p.a_tot[d][1] = a1[d];
  }
  predict(p, dt_code, scale, pos, vel);
}

double abyss_host_time_step_reg(const double *df12, double eta) {
  double df[3][4];
  std::memcpy(df, df12, sizeof(df));
  return new_step_reg(df, eta);
}

double abyss_host_time_step_irr(const double *f12, const double *df12, double eta) {
  double f[3][4], df[3][4];
  std::memcpy(f, f12, sizeof(f));
  std::memcpy(df, df12, sizeof(df));
  return new_step_irr(f, df, eta);
}

void abyss_host_block_time_step(double dt, double scale, int time_block, int *level,
                                unsigned long long *block, double *step) {
  abyss_ac tmp;
  tmp.scale = scale;
  tmp.time_block = time_block;
  int lv;
  ULL bl;
  double st;
  block_step(&tmp, dt, lv, bl, st);
  *level = lv;
  *block = bl;
  *step = st;
}

int abyss_host_regular_correct(int n, const double *x, const double *v, const double *a_tot,
                               const double *t0, const double *mass, double eps2, double new_time,
                               double scale, int i, double dt_reg, const double *a_reg_i, int n_old,
                               const int *old_nb, int n_new, const int *new_nb, const double *acc,
                               const double *jerk, const double *acc_irr, const double *jerk_irr,
                               double *new_pos, double *new_vel, double *a_reg_out,
                               double *a_tot_out) {
  if (n <= 0 || i < 0 || i >= n || n_old < 0 || n_new < 0) return ABYSS_ERR_ARG;
  auto star = [&](int j) {
    Star q{};
    for (int d = 0; d < 3; ++d) {
      q.x[d] = x[3 * (size_t)j + d];
      q.v[d] = v[3 * (size_t)j + d];
      for (int o = 0; o < 4; ++o) q.a_tot[d][o] = a_tot[12 * (size_t)j + 4 * d + o];
    }
    return q;
  };
  const Star self = star(i);
  double pos[3], vel[3];
  predict(self, n_old == 0 ? dt_reg : 0.0, scale, pos, vel);
  auto pred = [&](int j, double pj[3], double vj[3]) {
    const Star q = star(j);
    predict(q, new_time - t0[j], scale, pj, vj);
  };
  auto mfun = [&](int j) { return mass[j]; };
  double a_tmp[3] = {0, 0, 0}, adot_tmp[3] = {0, 0, 0};
  neighbour_change(old_nb, n_old, new_nb, n_new, pred, mfun, eps2, pos, vel, a_tmp, adot_tmp);
  double a_reg[3][4], a_irr[3][4], at[3][4], a2[3], a3[3];
  std::memcpy(a_reg, a_reg_i, sizeof(a_reg));
  std::memcpy(at, a_tot + 12 * (size_t)i, sizeof(at));
  std::memset(a_irr, 0, sizeof(a_irr));
  hermite_regular(pos, vel, a_reg, acc, jerk, a_tmp, adot_tmp, dt_reg * scale, new_pos, new_vel, a2, a3);
  commit_derivatives(acc, jerk, acc_irr, jerk_irr, a2, a3, n_new, a_reg, a_irr, at);
  std::memcpy(a_reg_out, a_reg, sizeof(a_reg));
  std::memcpy(a_tot_out, at, sizeof(at));
  return ABYSS_OK;
}

int abyss_host_irregular_steps(int n, const double *x, const double *v, const double *mass,
                               const double *a_tot, const double *a_reg, const double *a_irr,
                               const double *t_reg, const double *t_irr, const double *dt_irr,
                               const int *nnb, const int *nb, int nb_stride, double eps2, double scale,
                               int count, const int *idx, double *new_pos, double *new_vel,
                               double *a_irr_out, double *a_tot_out) {
  if (n <= 0 || count < 0 || nb_stride < 0 || !x || !v || !mass || !a_tot || !a_reg || !a_irr || !t_reg ||
      !t_irr || !dt_irr || !nnb || (count > 0 && (!idx || !new_pos || !new_vel || !a_irr_out || !a_tot_out)))
    return ABYSS_ERR_ARG;
  // the integrator's own state, so that the step runs through its own code
  // (the neighbour mirror included)
  abyss_ac tmp;
  tmp.n = n;
  tmp.scale = scale;
  tmp.p.eps2 = eps2;
  tmp.s.resize(n);
  for (int i = 0; i < n; ++i) {
    Star &p = tmp.s[i];
    for (int d = 0; d < 3; ++d) {
      p.x[d] = x[3 * (size_t)i + d];
      p.v[d] = v[3 * (size_t)i + d];
    }
    std::memcpy(p.a_tot, a_tot + 12 * (size_t)i, sizeof(p.a_tot));
    std::memcpy(p.a_reg, a_reg + 12 * (size_t)i, sizeof(p.a_reg));
    std::memcpy(p.a_irr, a_irr + 12 * (size_t)i, sizeof(p.a_irr));
    p.m = mass[i];
    p.t_reg = t_reg[i];
    p.t_irr = t_irr[i];
    p.dt_irr = dt_irr[i];
    if (nnb[i] < 0 || nnb[i] > nb_stride || (nnb[i] > 0 && !nb)) return ABYSS_ERR_ARG;
    p.nb.assign(nb + (size_t)i * nb_stride, nb + (size_t)i * nb_stride + nnb[i]);
    for (int j : p.nb)
      if (j < 0 || j >= n || j == i) return ABYSS_ERR_ARG;
  }
  build_slots(&tmp);
  for (int i = 0; i < n; ++i) put_rec(&tmp, i);
  Pending out;
  for (int k = 0; k < count; ++k) {
    const int i = idx[k];
    if (i < 0 || i >= n) return ABYSS_ERR_ARG;
    irregular_one(&tmp, i, out);
    const Star &p = tmp.s[i];
    for (int d = 0; d < 3; ++d) {
      new_pos[3 * (size_t)k + d] = out.move ? out.new_x[d] : p.x[d];
      new_vel[3 * (size_t)k + d] = out.move ? out.new_v[d] : p.v[d];
    }
    std::memcpy(a_irr_out + 12 * (size_t)k, out.a_irr, sizeof(out.a_irr));
    std::memcpy(a_tot_out + 12 * (size_t)k, out.a_tot, sizeof(out.a_tot));
  }
  return ABYSS_OK;
}

int abyss_host_time_level_irr(double scale, int time_block, double eta, int has_nb, const double *a_tot,
                              const double *a_irr, unsigned long long new_cur_irr, unsigned long long cur_reg,
                              unsigned long long tb_reg, int lv_reg, int *lv_irr, double *dt_irr,
                              unsigned long long *tb_irr) {
  if (!a_tot || !a_irr || !lv_irr || !dt_irr || !tb_irr) return ABYSS_ERR_ARG;
  abyss_ac tmp;
  tmp.scale = scale;
  tmp.time_block = time_block;
  tmp.p.eta_irr = eta;
  double at[3][4], ai[3][4];
  std::memcpy(at, a_tot, sizeof(at));
  std::memcpy(ai, a_irr, sizeof(ai));
  int lv = *lv_irr;
  double dt = *dt_irr;
  ULL tb = *tb_irr;
  int rc = ABYSS_OK;
  try {
    time_step_irr_of(&tmp, has_nb != 0, at, ai, new_cur_irr, cur_reg, tb_reg, lv_reg, lv, dt, tb);
  } catch (const std::exception &) {
    rc = ABYSS_ERR_STATE;
  }
  *lv_irr = lv;
  *dt_irr = dt;
  *tb_irr = tb;
  return rc;
}

int abyss_host_time_level_reg(double scale, int time_block, unsigned long long block_max, double eta,
                              int has_nb, const double *a_reg, double t_reg, unsigned long long cur_reg,
                              int *lv_reg, double *dt_reg, unsigned long long *tb_reg, int *lv_irr) {
  if (!a_reg || !lv_reg || !dt_reg || !tb_reg || !lv_irr) return ABYSS_ERR_ARG;
  abyss_ac tmp;
  tmp.scale = scale;
  tmp.time_block = time_block;
  tmp.block_max = block_max;
  tmp.p.eta_reg = eta;
  Star p{};
  std::memcpy(p.a_reg, a_reg, sizeof(p.a_reg));
  if (has_nb) p.nb.assign(1, 0);
  p.t_reg = t_reg;
  p.cur_reg = cur_reg;
  p.lv_reg = *lv_reg;
  p.dt_reg = *dt_reg;
  p.tb_reg = *tb_reg;
  p.lv_irr = *lv_irr;
  int rc = ABYSS_OK;
  try {
    time_step_reg(&tmp, p);
  } catch (const std::exception &) {
    rc = ABYSS_ERR_STATE;
  }
  *lv_reg = p.lv_reg;
  *dt_reg = p.dt_reg;
  *tb_reg = p.tb_reg;
  *lv_irr = p.lv_irr;
  return rc;
}

void abyss_host_initial_time_steps(double scale, int time_block, unsigned long long block_max, double eta_reg,
                                   double eta_irr, int has_nb, const double *a_tot, const double *a_reg,
                                   const double *a_irr, int *lv_reg, double *dt_reg, unsigned long long *tb_reg,
                                   int *lv_irr, double *dt_irr, unsigned long long *tb_irr) {
  abyss_ac tmp;
  tmp.scale = scale;
  tmp.time_block = time_block;
  tmp.block_max = block_max;
  tmp.p.eta_reg = eta_reg;
  tmp.p.eta_irr = eta_irr;
  Star p{};
  std::memcpy(p.a_tot, a_tot, sizeof(p.a_tot));
  std::memcpy(p.a_reg, a_reg, sizeof(p.a_reg));
  std::memcpy(p.a_irr, a_irr, sizeof(p.a_irr));
  if (has_nb) p.nb.assign(1, 0);
  init_time_step(&tmp, p);
  *lv_reg = p.lv_reg;
  *dt_reg = p.dt_reg;
  *tb_reg = p.tb_reg;
  *lv_irr = p.lv_irr;
  *dt_irr = p.dt_irr;
  *tb_irr = p.tb_irr;
}

double abyss_host_update_radius(double r2nb, int nnb, int fix_nb, int nb_max) {
  abyss_ac tmp;
  tmp.p.fix_nb = fix_nb;
  tmp.p.nb_max = nb_max;
  Star p{};
  p.nb.resize(nnb > 0 ? nnb : 0);
  p.r2nb = r2nb;
  update_radius(&tmp, p);
  return p.r2nb;
}

}  // extern "C"

// ------------------------------------------------------------------ state I/O

namespace {

constexpr char kCkptMagic[8] = {'A', 'B', 'Y', 'S', 'S', 'A', 'C', 'K'};
constexpr unsigned kCkptVersion = 1;

// Units of the reference's text files (src_mpi/def.h:51-60 and
// particle.h:204-214): input positions in kpc, velocities in km/s, masses in
// 1e9 Msun; output in pc, km/s and Msun; code units are G = 1.
constexpr double kPc = 3.08567758149137e18;
constexpr double kYr = 3.1536e7;
constexpr double kPositionUnit = 4.0;       // pc
constexpr double kVelocityUnit = 4e-10;     // pc / yr
constexpr double kMassUnit = 0.0001424198;  // Msun

template <class T>
void put(std::ofstream &f, const T &v) {
  f.write(reinterpret_cast<const char *>(&v), sizeof(T));
}
template <class T>
bool get(std::ifstream &f, T &v) {
  return (bool)f.read(reinterpret_cast<char *>(&v), sizeof(T));
}

}  // namespace

namespace {
int load_body(std::ifstream &f, abyss_ctx *ctx, int n, int threads, abyss_ac **out);
}  // namespace

extern "C" {

int abyss_ac_save(const abyss_ac *ac, const char *path) {
  if (!ac || !path) return ABYSS_ERR_ARG;
  if (ac->in_block) return ABYSS_ERR_STATE;  // only between regular blocks
  const int rs = resident_sync_host(ac);
  if (rs != ABYSS_OK) return rs;
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) return ABYSS_ERR_ARG;
  f.write(kCkptMagic, sizeof(kCkptMagic));
  put(f, kCkptVersion);
  put(f, (unsigned)sizeof(Star::a_tot));
  put(f, ac->n);
  put(f, ac->p);
  put(f, ac->scale);
  put(f, ac->time_block);
  put(f, ac->block_max);
  put(f, ac->time_step);
  put(f, ac->next_reg_block);
  put(f, (int)ac->done);
  put(f, ac->st);
  for (const Star &p : ac->s) {
    put(f, p.x);
    put(f, p.v);
    put(f, p.m);
    put(f, p.a_tot);
    put(f, p.a_reg);
    put(f, p.a_irr);
    put(f, p.r2nb);
    put(f, p.t_reg);
    put(f, p.t_irr);
    put(f, p.dt_reg);
    put(f, p.dt_irr);
    const ULL u[6] = {p.cur_reg, p.cur_irr, p.new_cur_irr, p.next_irr, p.tb_reg, p.tb_irr};
    put(f, u);
    put(f, p.lv_reg);
    put(f, p.lv_irr);
    put(f, (int)p.nb.size());
    if (!p.nb.empty()) f.write(reinterpret_cast<const char *>(p.nb.data()), sizeof(int) * p.nb.size());
  }
  f.write(kCkptMagic, sizeof(kCkptMagic));  // trailer: the file is complete
  return f ? ABYSS_OK : ABYSS_ERR_STATE;
}

int abyss_ac_load(abyss_ctx *ctx, const char *path, int threads, abyss_ac **out) {
  if (!path || !out || threads < 0) return ABYSS_ERR_ARG;  // a null ctx: host-side calls only
  std::ifstream f(path, std::ios::binary);
  if (!f) return ABYSS_ERR_ARG;
  char magic[8];
  unsigned version = 0, dsz = 0;
  int n = 0;
  if (!f.read(magic, 8) || std::memcmp(magic, kCkptMagic, 8) != 0) return ABYSS_ERR_STATE;
  if (!get(f, version) || version != kCkptVersion || !get(f, dsz) || dsz != sizeof(Star::a_tot)) return ABYSS_ERR_STATE;
  if (!get(f, n) || n < 2) return ABYSS_ERR_STATE;
  // the bytes left bound the particle count that the file may claim, so that
  // a damaged count is refused before anything is allocated for it
  constexpr long long kMinRecord = sizeof(Star::x) + sizeof(Star::v) + sizeof(Star::m) + 3 * sizeof(Star::a_tot) +
                                   5 * sizeof(double) + 6 * sizeof(ULL) + 3 * sizeof(int);
  const std::streampos here = f.tellg();
  f.seekg(0, std::ios::end);
  const long long left = (long long)(f.tellg() - here);
  f.seekg(here);
  if (!f || (long long)n > left / kMinRecord) return ABYSS_ERR_STATE;
  return load_body(f, ctx, n, threads, out);
}

}  // extern "C"

namespace {

// The checkpoint after its header (n particles, within the file's size): the
// integrator, or an error; host allocation failure is ABYSS_ERR_OOM.
int load_body(std::ifstream &f, abyss_ctx *ctx, int n, int threads, abyss_ac **out) try {
  char magic[8];
  std::unique_ptr<abyss_ac> owner(new abyss_ac);
  abyss_ac *ac = owner.get();
  ac->ctx = ctx;
  ac->n = n;
  int done = 0;
  bool ok = get(f, ac->p) && get(f, ac->scale) && get(f, ac->time_block) && get(f, ac->block_max) &&
            get(f, ac->time_step) && get(f, ac->next_reg_block) && get(f, done) && get(f, ac->st);
  ac->done = done != 0;
  ac->p.threads = threads;
  // header fields in the range the integrator produces (abyss_ac_create's
  // parameter rule; block times of 2^time_block with time_block in [-62, -1]),
  // so that a damaged file cannot size buffers or shift block counts out of range
  const abyss_ac_params &q = ac->p;
  if (ok)
    ok = q.nb_max > 0 && q.nb_max <= (1 << 20) && q.fix_nb > 0 && q.fix_nb < q.nb_max && q.t_end > 0 &&
         std::isfinite(q.t_end) && q.eta_reg > 0 && q.eta_irr > 0 && q.eps2 >= 0 && std::isfinite(q.eps2) &&
         ac->scale > 0 && std::isfinite(ac->scale) && ac->time_block >= -62 && ac->time_block <= -1 &&
         ac->block_max == pow2_blocks(-ac->time_block) && ac->time_step == pow2(ac->time_block) &&
         ac->next_reg_block <= ac->block_max;
  const int lv_lo = ac->time_block, lv_hi = ac->time_block + 62;
  if (ok) ac->s.resize(n);
  for (int i = 0; ok && i < n; ++i) {
    Star &p = ac->s[i];
    ULL u[6];
    int nn = 0;
    ok = get(f, p.x) && get(f, p.v) && get(f, p.m) && get(f, p.a_tot) && get(f, p.a_reg) && get(f, p.a_irr) &&
         get(f, p.r2nb) && get(f, p.t_reg) && get(f, p.t_irr) && get(f, p.dt_reg) && get(f, p.dt_irr) &&
         get(f, u) && get(f, p.lv_reg) && get(f, p.lv_irr) && get(f, nn) && nn >= 0 && nn <= n;
    if (ok)
      ok = p.lv_reg >= lv_lo && p.lv_reg <= lv_hi && p.lv_irr >= lv_lo && p.lv_irr <= lv_hi && p.r2nb >= 0 &&
           std::isfinite(p.r2nb) && std::isfinite(p.m);
    if (!ok) break;
    p.cur_reg = u[0];
    p.cur_irr = u[1];
    p.new_cur_irr = u[2];
    p.next_irr = u[3];
    p.tb_reg = u[4];
    p.tb_irr = u[5];
    p.nb.resize(nn);
    if (nn > 0) ok = (bool)f.read(reinterpret_cast<char *>(p.nb.data()), sizeof(int) * (size_t)nn);
    for (int j : p.nb)
      if (j < 0 || j >= n) ok = false;
  }
  if (ok) ok = f.read(magic, 8) && std::memcmp(magic, kCkptMagic, 8) == 0;
  if (!ok) return ABYSS_ERR_STATE;
  *out = owner.release();
  return ABYSS_OK;
} catch (const std::bad_alloc &) {
  return ABYSS_ERR_OOM;
}

}  // namespace

extern "C" {

int abyss_ac_write_snapshot(const abyss_ac *ac, const char *path, double output_time, double output_time_step) {
  if (!ac || !path) return ABYSS_ERR_ARG;
  const int rs = resident_sync_host(ac);
  if (rs != ABYSS_OK) return rs;
  std::ofstream f(path, std::ios::trunc);
  if (!f) return ABYSS_ERR_ARG;
  const double now = ac->next_reg_block * ac->time_step;  // code time of the state
  const int w = 18;
  f << now * ac->scale * 1e10 / 1e6 << " Myr, " << "\n";
  f << output_time << ", " << output_time_step << ", " << now << "\n";
  f << std::left << std::setw(w) << "PID" << std::setw(w) << "Mass (Msun)" << std::setw(w) << "X (pc)"
    << std::setw(w) << "Y (pc)" << std::setw(w) << "Z (pc)" << std::setw(w) << "Vx (km/s)" << std::setw(w)
    << "Vy (km/s)" << std::setw(w) << "Vz (km/s)" << "\n";
  auto kms = [](double u) { return u * kVelocityUnit / kYr * kPc / 1e5; };  // ReadWrite.cpp:257-264 order
  for (int i = 0; i < ac->n; ++i) {
    const Star &p = ac->s[i];
    double pos[3], vel[3];
    predict(p, now - p.t_irr, ac->scale, pos, vel);
    f << std::left << std::fixed << std::setprecision(8) << std::setw(w) << i << std::setw(w) << p.m * kMassUnit
      << std::setw(w) << pos[0] * kPositionUnit << std::setw(w) << pos[1] * kPositionUnit << std::setw(w)
      << pos[2] * kPositionUnit << std::setw(w) << kms(vel[0]) << std::setw(w) << kms(vel[1]) << std::setw(w)
      << kms(vel[2]) << '\n';
  }
  return f ? ABYSS_OK : ABYSS_ERR_STATE;
}

int abyss_read_reference_ic(const char *path, int *n, double *x, double *v, double *mass) {
  if (!path || !n) return ABYSS_ERR_ARG;
  std::ifstream f(path);
  if (!f) return ABYSS_ERR_ARG;
  std::string line;
  int row = 0;
  while (std::getline(f, line)) {
    if (x && v && mass) {
      if (row >= *n) return ABYSS_ERR_ARG;
      double d[7] = {0, 0, 0, 0, 0, 0, 0};
      std::istringstream iss(line);
      double val;
      int col = 0;
      while (col < 7 && iss >> val) d[col++] = val;
      for (int k = 0; k < 3; ++k) {
        x[3 * (size_t)row + k] = d[k] * 1000 / kPositionUnit;
        v[3 * (size_t)row + k] = d[3 + k] * (1e5 * kYr / kPc) / kVelocityUnit;
      }
      mass[row] = d[6] * 1e9 / kMassUnit;
    }
    ++row;
  }
  if (x && v && mass && row != *n) return ABYSS_ERR_ARG;
  *n = row;
  return ABYSS_OK;
}

}  // extern "C"
