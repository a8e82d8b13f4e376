/* abyss_host.h -- the host integrator's per-particle rules (libabyss_reg.so),
 * exported so that they can be checked against the reference without a GPU.
 * Arrays [3][4] are row-major (dimension, derivative order) as in
 * src_mpi/particle.h:37-39. */
#ifndef ABYSS_HOST_H
#define ABYSS_HOST_H
#ifdef __cplusplus
extern "C" {
#endif

/* predictParticleSecondOrder, src_mpi/Particle/UpdateParticle.cpp:37-59. */
void abyss_host_predict(const double *x, const double *v, const double *a0, const double *a1,
                        double dt_code, double scale, double *pos, double *vel);
/* getNewTimeStepReg, src_mpi/TimeStepRoutines.cpp:10-25. */
double abyss_host_time_step_reg(const double *df12, double eta);
/* getNewTimeStepIrr, src_mpi/TimeStepRoutines.cpp:28-63. */
double abyss_host_time_step_irr(const double *f12, const double *df12, double eta);
/* getBlockTimeStep, src_mpi/TimeStepRoutines.cpp:102-115. */
void abyss_host_block_time_step(double dt, double scale, int time_block, int *level,
                                unsigned long long *block, double *step);
/* Particle::updateRegularParticleCuda (src_mpi/Particle/ComputeAcceleration.cpp:
 * 405-661) for particle i of an n-particle state (x, v [n][3], a_tot [n][3][4],
 * t0 = time each particle was last advanced to), given the GPU's new list and
 * regular acc/jerk and the irregular acc/jerk over the new list.  Writes the
 * corrected position/velocity and the new a_reg, a_tot [3][4]. */
int abyss_host_regular_correct(int n, const double *x, const double *v, const double *a_tot,
                               const double *t0, const double *mass, double eps2, double new_time,
                               double scale, int i, double dt_reg, const double *a_reg_i, int n_old,
                               const int *old_nb, int n_new, const int *new_nb, const double *acc,
                               const double *jerk, const double *acc_irr, const double *jerk_irr,
                               double *new_pos, double *new_vel, double *a_reg_out,
                               double *a_tot_out);

#ifdef __cplusplus
}
#endif
#endif
