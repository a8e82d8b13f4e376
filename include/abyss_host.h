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
/* Particle::computeAccelerationIrr (src_mpi/Particle/ComputeAcceleration.cpp:14-190)
 * for the `count` particles idx[k] of an n-particle state, each from the same
 * pre-step state of all others (one irregular level of the integrator).
 * Per particle: x, v [n][3]; mass, t_reg, t_irr, dt_irr [n] (CurrentTimeReg,
 * CurrentTimeIrr, TimeStepIrr in code time); a_tot, a_reg, a_irr [n][3][4];
 * nnb[n] neighbours in rows of nb_stride.  Writes, per listed particle k, the
 * new position/velocity [count][3] and the new a_irr, a_tot [count][3][4].  A
 * particle without neighbours keeps its position and derivatives, as in the
 * reference.  The position correction uses dt^5 where the reference's line 162
 * reads an uninitialised variable. */
int abyss_host_irregular_steps(int n, const double *x, const double *v, const double *mass,
                               const double *a_tot, const double *a_reg, const double *a_irr,
                               const double *t_reg, const double *t_irr, const double *dt_irr,
                               const int *nnb, const int *nb, int nb_stride, double eps2, double scale,
                               int count, const int *idx, double *new_pos, double *new_vel,
                               double *a_irr_out, double *a_tot_out);
/* Particle::calculateTimeStepIrr (src_mpi/Particle/UpdateParticle.cpp:151-241):
 * the new irregular level from the particle's new a_tot, a_irr [3][4] and its
 * blocks (NewCurrentBlockIrr, CurrentBlockReg, TimeBlockReg, TimeLevelReg).
 * lv_irr, dt_irr, tb_irr hold TimeLevelIrr, TimeStepIrr, TimeBlockIrr on entry
 * and on return.  ABYSS_ERR_STATE where the reference throws (step > 1). */
int abyss_host_time_level_irr(double scale, int time_block, double eta, int has_nb, const double *a_tot,
                              const double *a_irr, unsigned long long new_cur_irr, unsigned long long cur_reg,
                              unsigned long long tb_reg, int lv_reg, int *lv_irr, double *dt_irr,
                              unsigned long long *tb_irr);
/* Particle::calculateTimeStepReg (src_mpi/Particle/UpdateParticle.cpp:314-407):
 * the new regular level from a_reg [3][4], CurrentTimeReg and CurrentBlockReg.
 * lv_reg, dt_reg, tb_reg (TimeLevelReg, TimeStepReg, TimeBlockReg) and lv_irr
 * (TimeLevelIrr, set to the regular level when has_nb is 0) are updated in
 * place.  ABYSS_ERR_STATE where the reference throws. */
int abyss_host_time_level_reg(double scale, int time_block, unsigned long long block_max, double eta,
                              int has_nb, const double *a_reg, double t_reg, unsigned long long cur_reg,
                              int *lv_reg, double *dt_reg, unsigned long long *tb_reg, int *lv_irr);
/* Particle::initializeTimeStep (src_mpi/Particle/Initialize.cpp:199-230): the
 * first regular and irregular levels, steps and blocks from the initial
 * a_tot, a_reg, a_irr [3][4] (eta_reg and eta_irr both the reference's eta). */
void abyss_host_initial_time_steps(double scale, int time_block, unsigned long long block_max, double eta_reg,
                                   double eta_irr, int has_nb, const double *a_tot, const double *a_reg,
                                   const double *a_irr, int *lv_reg, double *dt_reg, unsigned long long *tb_reg,
                                   int *lv_irr, double *dt_irr, unsigned long long *tb_irr);
/* Particle::updateRadius (src_mpi/Particle/UpdateParticle.cpp:108-139): the new
 * squared neighbour radius after a regular step that found nnb neighbours,
 * FixNumNeighbor and NumNeighborMax given as fix_nb and nb_max. */
double abyss_host_update_radius(double r2nb, int nnb, int fix_nb, int nb_max);

#ifdef __cplusplus
}
#endif
#endif
