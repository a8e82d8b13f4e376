/* Test infrastructure only: the CPU oracle (checker) for the Ahmad-Cohen
 * regular-force path.  Nothing in the product links or calls this; only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg do.
 *
 * A plain-C FP64 restatement of the reference's CPU algorithm:
 *   predictor          src_mpi/Particle/UpdateParticle.cpp:37-59
 *   regular force      src_mpi/Particle/ComputeAcceleration.cpp:235-299
 *   Hermite corrector  src_mpi/Particle/ComputeAcceleration.cpp:604-636
 *   timestep rules     src_mpi/TimeStepRoutines.cpp:10-25, 28-63, 102-115
 * with one documented extension: Plummer softening eps^2 is added to r^2 in
 * the force terms only (as src/Particle/CalculateRegForce.cpp:21 does); the
 * neighbour test stays on the unsoftened r^2 < R_nb^2.  With eps2 == 0 the
 * arithmetic is operation-for-operation the reference's, and the tests pin
 * it bit-exactly against the reference compiled from its own sources
 * (oracle/_ref) and against the committed golden vectors (tests/golden).
 *
 * Arrays are row-major: positions [n][3], per-target lists [nt][cap].
 */
#ifndef ABYSS_ORACLE_H
#define ABYSS_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Second-order prediction of every particle to new_time
 * (UpdateParticle.cpp:37-59): dt = (new_time - t0[j]) * time_scale,
 * x_p = ((a1 dt/3 + a0) dt/2 + v) dt + x,  v_p = (a1 dt/2 + a0) dt + v;
 * dt == 0 copies x, v. */
void oracle_predict(int n, const double *x, const double *v, const double *a0,
                    const double *a1, const double *t0, double new_time,
                    double time_scale, double *px, double *pv);

/* Regular/irregular split for each target (ComputeAcceleration.cpp:235-299):
 * for every j != target in ascending index order, r2 = |x_j - x_i|^2;
 * r2 < r2nb[i] -> j is appended to the target's new neighbour list and its
 * acc/jerk go to the irregular part; otherwise to the regular part.
 * Lists longer than cap are truncated; nnb holds the true count.
 * Returns the number of targets whose list overflowed. */
int oracle_reg_force(int n, const double *px, const double *pv, const double *mass,
                     const double *r2nb, double eps2, int nt, const int *targets,
                     int cap, double *acc_reg, double *jerk_reg, double *acc_irr,
                     double *jerk_irr, int *nnb, int *list, int nthreads);

/* The same sums for a bounded sample: targets[0..nt) against j in [j0, j1)
 * only (self and neighbour handling unchanged).  Used to time the CPU
 * baseline on a sample of a large workload. */
void oracle_reg_force_range(int n, const double *px, const double *pv, const double *mass,
                            const double *r2nb, double eps2, int nt, const int *targets,
                            int j0, int j1, double *acc_reg, double *jerk_reg, int *nnb,
                            int nthreads);

/* Fourth-order Hermite corrector of one particle after a regular step
 * (ComputeAcceleration.cpp:604-636).  a_reg_old = old regular (acc, jerk)
 * [3][2]; a_new/adot_new = new regular; a_tmp/adot_tmp = neighbour-change
 * correction; dt = step in code time.  Writes new position/velocity and the
 * second/third derivatives a2, a3 [3]. */
void oracle_hermite_correct(const double *pos, const double *vel, const double *a_reg_old,
                            const double *a_new, const double *adot_new, const double *a_tmp,
                            const double *adot_tmp, double dt, double *new_pos,
                            double *new_vel, double *a2, double *a3);

/* Aarseth criteria (TimeStepRoutines.cpp:10-25 and 28-63); df, f are [3][4]. */
double oracle_time_step_reg(const double *v, const double *df, double eta);
double oracle_time_step_irr(const double *f, const double *df, double eta);

/* Power-of-two quantisation (TimeStepRoutines.cpp:102-115). */
void oracle_block_time_step(double dt, double time_scale, int time_block, int *level,
                            unsigned long long *block, double *step);

/* Per-target sums of the magnitudes of the regular acc and jerk terms (the
 * natural error scale of an FP32 pair sum). */
void oracle_reg_scale(int n, const double *px, const double *pv, const double *mass,
                      const double *r2nb, double eps2, int nt, const int *targets,
                      double *acc_abs, double *jerk_abs, int nthreads);

/* Total energy T + W (FP64, softened potential) of n particles. */
/* Second and third derivatives of the acceleration at a common time, split into
 * regular (r^2 >= R^2, unsoftened) and irregular parts: CalculateAcceleration23
 * (src_mpi/Particle/Initialize.cpp:102-185) in its operation order, j ascending,
 * with eps2 added to r^2 in the force terms.  x, v, a0, a1: [n][3]; targets
 * [nt]; outputs [nt][3].  With eps2 = 0 it equals the reference except for a
 * pair at exactly r^2 = R^2 (the reference counts it irregular). */
void oracle_init_derivs23(int n, const double *x, const double *v, const double *mass,
                          const double *r2nb, const double *a0, const double *a1, double eps2,
                          int nt, const int *targets, double *reg2, double *reg3, double *irr2,
                          double *irr3, int nthreads);

double oracle_energy(int n, const double *x, const double *v, const double *mass,
                     double eps2, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
