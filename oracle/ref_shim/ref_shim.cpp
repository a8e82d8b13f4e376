// Test infrastructure only (the checker, never the product).
//
// C entry points around the reference's own, unmodified single-particle
// physics (compiled from src_mpi/Particle/{ComputeAcceleration,UpdateParticle,
// Initialize}.cpp and src_mpi/TimeStepRoutines.cpp by oracle/Makefile), so
// that tests can run the reference's CPU regular force, corrector, predictor
// and timestep rules on arrays.  The globals below are the six symbols those
// files leave undefined (src_mpi/global.h:12,34,38,58,68 and time_block).
//
// Parallel runs mirror the reference's MPI worker farm
// (src_mpi/WorkerRoutines.cpp:66-74: one particle per RegForce task) with
// host threads: computeAccelerationReg() writes only to its own particle and
// reads the others, so distinct particles may run concurrently.
#include <thread>
#include <vector>
#include <atomic>
#include <cstring>
#include "global.h"

Particle *particles = nullptr;
GlobalVariable *global_variable = nullptr;
int *ActiveIndexToOriginalIndex = nullptr;
double EnzoTimeStep = 1.0;
int time_block = 0;
ULL block_max = 1;

void CalculateAcceleration01(Particle *ptcl);
void CalculateAcceleration23(Particle *ptcl);
double getNewTimeStepReg(double v[3], double df[3][4]);
double getNewTimeStepIrr(double f[3][4], double df[3][4]);
double getNewTimeStep(double f[3][4], double df[3][4]);
void getBlockTimeStep(double dt, int &TimeLevel, ULL &TimeBlock, double &TimeStep);

static int g_n = 0;

template <class F>
static void parallel_over(int count, int nthreads, F &&f) {
    if (nthreads <= 1 || count < 2) {
        for (int k = 0; k < count; ++k) f(k);
        return;
    }
    std::atomic<int> next(0);
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t)
        pool.emplace_back([&]() {
            for (;;) {
                int k = next.fetch_add(1);
                if (k >= count) break;
                f(k);
            }
        });
    for (auto &th : pool) th.join();
}

extern "C" {

int ref_particle_bytes(void) { return (int)sizeof(Particle); }
int ref_max_neighbors(void) { return MaxNumberOfNeighbor; }
int ref_num_neighbor_max(void) { return NumNeighborMax; }
int ref_fix_num_neighbor(void) { return FixNumNeighbor; }
double ref_eta(void) { return eta; }

int ref_alloc(int n) {
    delete[] particles;
    delete global_variable;
    delete[] ActiveIndexToOriginalIndex;
    particles = new Particle[n];
    global_variable = new GlobalVariable;
    global_variable->LastParticleIndex = n - 1;
    global_variable->next_time = 0.0;
    ActiveIndexToOriginalIndex = new int[n];
    for (int i = 0; i < n; ++i) {
        ActiveIndexToOriginalIndex[i] = i;
        particles[i].PID = i;
        particles[i].ParticleIndex = i;
        particles[i].isActive = true;
    }
    g_n = n;
    return 0;
}

// One line of the reference's input file through its own Particle::initialize
// and normalizeParticle (particle.h:139-147,204-214): code-unit x, v, mass.
void ref_particle_from_row(const double *row7, double *x, double *v, double *mass) {
    Particle p;
    double d[7];
    std::memcpy(d, row7, sizeof(d));
    p.initialize(d, 0);
    p.normalizeParticle();
    for (int k = 0; k < 3; ++k) {
        x[k] = p.Position[k];
        v[k] = p.Velocity[k];
    }
    *mass = p.Mass;
}

void ref_free(void) {
    delete[] particles;
    delete global_variable;
    delete[] ActiveIndexToOriginalIndex;
    particles = nullptr;
    global_variable = nullptr;
    ActiveIndexToOriginalIndex = nullptr;
    g_n = 0;
}

void ref_set_globals(double enzo_time_step, int tblock, unsigned long long bmax) {
    EnzoTimeStep = enzo_time_step;
    time_block = tblock;
    block_max = bmax;
}

// Per-particle state.  a_* are [3][4] row-major (dim, order) as in
// src_mpi/particle.h:37-39.
void ref_set_particle(int i, const double *x, const double *v, double mass, double r2nb,
                      const double *a_tot, const double *a_reg, const double *a_irr,
                      double t_reg, double t_irr, double dt_reg, double dt_irr,
                      int nnb, const int *nb) {
    Particle &p = particles[i];
    for (int d = 0; d < 3; ++d) {
        p.Position[d] = x[d];
        p.Velocity[d] = v[d];
        for (int o = 0; o < 4; ++o) {
            p.a_tot[d][o] = a_tot[d * 4 + o];
            p.a_reg[d][o] = a_reg[d * 4 + o];
            p.a_irr[d][o] = a_irr[d * 4 + o];
        }
    }
    p.Mass = mass;
    p.RadiusOfNeighbor = r2nb;
    p.CurrentTimeReg = t_reg;
    p.CurrentTimeIrr = t_irr;
    p.TimeStepReg = dt_reg;
    p.TimeStepIrr = dt_irr;
    p.NumberOfNeighbor = nnb;
    for (int k = 0; k < nnb; ++k) p.Neighbors[k] = nb[k];
}

// Bulk form of ref_set_particle for large particle sets: x, v, a_tot [n][3][..]
// arrays as in ref_set_particle; every particle gets no neighbour list, the
// given times and steps, and zero regular/irregular derivatives.
void ref_set_all(int n, const double *x, const double *v, const double *mass, const double *r2nb,
                 const double *a_tot, const double *t_reg, const double *t_irr,
                 const double *dt_reg) {
    for (int i = 0; i < n; ++i) {
        Particle &p = particles[i];
        for (int d = 0; d < 3; ++d) {
            p.Position[d] = x[3 * (size_t)i + d];
            p.Velocity[d] = v[3 * (size_t)i + d];
            for (int o = 0; o < 4; ++o) {
                p.a_tot[d][o] = a_tot[12 * (size_t)i + 4 * d + o];
                p.a_reg[d][o] = 0.0;
                p.a_irr[d][o] = 0.0;
            }
        }
        p.Mass = mass[i];
        p.RadiusOfNeighbor = r2nb[i];
        p.CurrentTimeReg = t_reg[i];
        p.CurrentTimeIrr = t_irr[i];
        p.TimeStepReg = dt_reg[i];
        p.TimeStepIrr = dt_reg[i];
        p.NumberOfNeighbor = 0;
    }
}

void ref_set_blocks(int i, unsigned long long cur_reg, unsigned long long cur_irr,
                    unsigned long long tb_reg, unsigned long long tb_irr, int lvl_reg, int lvl_irr,
                    unsigned long long new_cur_irr) {
    Particle &p = particles[i];
    p.CurrentBlockReg = cur_reg;
    p.CurrentBlockIrr = cur_irr;
    p.TimeBlockReg = tb_reg;
    p.TimeBlockIrr = tb_irr;
    p.TimeLevelReg = lvl_reg;
    p.TimeLevelIrr = lvl_irr;
    p.NewCurrentBlockIrr = new_cur_irr;
}

void ref_get_blocks(int i, unsigned long long *out_ull4, int *out_lvl2, double *out_dt2) {
    Particle &p = particles[i];
    out_ull4[0] = p.CurrentBlockReg;
    out_ull4[1] = p.CurrentBlockIrr;
    out_ull4[2] = p.TimeBlockReg;
    out_ull4[3] = p.TimeBlockIrr;
    out_lvl2[0] = p.TimeLevelReg;
    out_lvl2[1] = p.TimeLevelIrr;
    out_dt2[0] = p.TimeStepReg;
    out_dt2[1] = p.TimeStepIrr;
}

void ref_get_particle(int i, double *x, double *v, double *a_tot, double *a_reg, double *a_irr,
                      double *newpos, double *newvel, double *r2nb, int *nnb, int *nb,
                      int *new_nnb, int *new_nb, int cap) {
    Particle &p = particles[i];
    for (int d = 0; d < 3; ++d) {
        x[d] = p.Position[d];
        v[d] = p.Velocity[d];
        newpos[d] = p.NewPosition[d];
        newvel[d] = p.NewVelocity[d];
        for (int o = 0; o < 4; ++o) {
            a_tot[d * 4 + o] = p.a_tot[d][o];
            a_reg[d * 4 + o] = p.a_reg[d][o];
            a_irr[d * 4 + o] = p.a_irr[d][o];
        }
    }
    *r2nb = p.RadiusOfNeighbor;
    *nnb = p.NumberOfNeighbor;
    for (int k = 0; k < p.NumberOfNeighbor && k < cap; ++k) nb[k] = p.Neighbors[k];
    *new_nnb = p.NewNumberOfNeighbor;
    for (int k = 0; k < p.NewNumberOfNeighbor && k < cap; ++k) new_nb[k] = p.NewNeighbors[k];
}

// Particle::computeAccelerationReg (ComputeAcceleration.cpp:197-398) for each idx.
void ref_compute_reg(int count, const int *idx, int nthreads) {
    parallel_over(count, nthreads, [&](int k) { particles[idx[k]].computeAccelerationReg(); });
}

// computeAccelerationReg for each idx with every other particle's state held
// at its value before the step.  The reference's own farm lets a RegForce task
// overwrite its particle's a_tot (ComputeAcceleration.cpp:340-341) while other
// tasks still predict that particle from a_tot (UpdateParticle.cpp:54-55), so
// its CPU results depend on task order; the GPU path predicts every particle
// first.  This runs the targets one at a time and restores each target's
// derivative state after copying its outputs, which gives the predict-first
// semantics.  Outputs: a_reg/a_irr/a_tot [k][3][4], new position/velocity
// [k][3], new list count and entries [k][cap].
void ref_compute_reg_isolated(int count, const int *idx, double *a_reg, double *a_irr,
                              double *a_tot, double *newpos, double *newvel, int *new_nnb,
                              int *new_nb, int cap) {
    for (int k = 0; k < count; ++k) {
        Particle &p = particles[idx[k]];
        double s_tot[3][4], s_reg[3][4], s_irr[3][4];
        std::memcpy(s_tot, p.a_tot, sizeof(s_tot));
        std::memcpy(s_reg, p.a_reg, sizeof(s_reg));
        std::memcpy(s_irr, p.a_irr, sizeof(s_irr));
        p.computeAccelerationReg();
        std::memcpy(a_reg + 12 * k, p.a_reg, sizeof(s_reg));
        std::memcpy(a_irr + 12 * k, p.a_irr, sizeof(s_irr));
        std::memcpy(a_tot + 12 * k, p.a_tot, sizeof(s_tot));
        for (int d = 0; d < 3; ++d) {
            newpos[3 * k + d] = p.NewPosition[d];
            newvel[3 * k + d] = p.NewVelocity[d];
        }
        new_nnb[k] = p.NewNumberOfNeighbor;
        for (int j = 0; j < p.NewNumberOfNeighbor && j < cap; ++j) new_nb[(long)k * cap + j] = p.NewNeighbors[j];
        std::memcpy(p.a_tot, s_tot, sizeof(s_tot));
        std::memcpy(p.a_reg, s_reg, sizeof(s_reg));
        std::memcpy(p.a_irr, s_irr, sizeof(s_irr));
    }
}

// Particle::computeAccelerationIrr (ComputeAcceleration.cpp:14-190) for each idx.
void ref_compute_irr(int count, const int *idx, int nthreads) {
    parallel_over(count, nthreads, [&](int k) { particles[idx[k]].computeAccelerationIrr(); });
}

// Particle::updateRegularParticleCuda (ComputeAcceleration.cpp:405-661).
// `list` holds active indices; it is copied because the reference rewrites it.
void ref_update_reg_cuda(int i, const int *list, int nnb, const double *new_a, const double *new_adot) {
    std::vector<int> tmp(list, list + nnb);
    double a[3] = {new_a[0], new_a[1], new_a[2]};
    double ad[3] = {new_adot[0], new_adot[1], new_adot[2]};
    particles[i].updateRegularParticleCuda(tmp.data(), nnb, a, ad);
}

// updateRegularParticleCuda for target i with the same predict-first semantics
// as ref_compute_reg_isolated: outputs are copied out, then the target's
// derivative state is restored so later targets see the pre-step state.
void ref_update_reg_cuda_isolated(int i, const int *list, int nnb, const double *new_a,
                                  const double *new_adot, double *a_reg, double *a_irr,
                                  double *a_tot, double *newpos, double *newvel) {
    Particle &p = particles[i];
    double s_tot[3][4], s_reg[3][4], s_irr[3][4];
    std::memcpy(s_tot, p.a_tot, sizeof(s_tot));
    std::memcpy(s_reg, p.a_reg, sizeof(s_reg));
    std::memcpy(s_irr, p.a_irr, sizeof(s_irr));
    ref_update_reg_cuda(i, list, nnb, new_a, new_adot);
    std::memcpy(a_reg, p.a_reg, sizeof(s_reg));
    std::memcpy(a_irr, p.a_irr, sizeof(s_irr));
    std::memcpy(a_tot, p.a_tot, sizeof(s_tot));
    for (int d = 0; d < 3; ++d) {
        newpos[d] = p.NewPosition[d];
        newvel[d] = p.NewVelocity[d];
    }
    std::memcpy(p.a_tot, s_tot, sizeof(s_tot));
    std::memcpy(p.a_reg, s_reg, sizeof(s_reg));
    std::memcpy(p.a_irr, s_irr, sizeof(s_irr));
}

// Particle::predictParticleSecondOrder, double overload (UpdateParticle.cpp:37-59).
void ref_predict(int i, double dt, double *pos, double *vel) {
    particles[i].predictParticleSecondOrder(dt, pos, vel);
}

// Particle::predictParticleSecondOrder, CUDA_REAL=float overload (UpdateParticle.cpp:13-35).
void ref_predict_f32(int i, double dt, float *pos, float *vel) {
    particles[i].predictParticleSecondOrder(dt, pos, vel);
}

void ref_update_particle(int i) { particles[i].updateParticle(); }
void ref_update_radius(int i) { particles[i].updateRadius(); }
void ref_time_step_reg(int i) { particles[i].calculateTimeStepReg(); }
void ref_time_step_irr(int i) { particles[i].calculateTimeStepIrr(); }
void ref_initialize_time_step(int i) { particles[i].initializeTimeStep(); }
void ref_init_acc01(int i) { CalculateAcceleration01(&particles[i]); }
void ref_init_acc23(int i) { CalculateAcceleration23(&particles[i]); }

double ref_new_time_step_reg(const double *v3, const double *df12) {
    double v[3] = {v3[0], v3[1], v3[2]};
    double df[3][4];
    std::memcpy(df, df12, sizeof(df));
    return getNewTimeStepReg(v, df);
}

double ref_new_time_step_irr(const double *f12, const double *df12) {
    double f[3][4], df[3][4];
    std::memcpy(f, f12, sizeof(f));
    std::memcpy(df, df12, sizeof(df));
    return getNewTimeStepIrr(f, df);
}

void ref_block_time_step(double dt, int *level, unsigned long long *block, double *step) {
    int lv = 0;
    ULL bl = 0;
    double st = 0;
    getBlockTimeStep(dt, lv, bl, st);
    *level = lv;
    *block = bl;
    *step = st;
}

}  // extern "C"
