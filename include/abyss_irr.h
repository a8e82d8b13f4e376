/* abyss_irr.h -- irregular steps on the GPU (libabyss_reg.so).
 *
 * The Ahmad-Cohen irregular force -- every particle due before the next
 * regular block, level by level in increasing block time -- run with its level
 * loop on the device, for an integration of include/abyss_ac.h.  Reference:
 * the IrrForce/IrrUpdate tasks (src_mpi/WorkerRoutines.cpp:46-64, 76-87)
 * dispatched level by level from src_mpi/RootRoutines.cpp:488-1005; per
 * particle computeAccelerationIrr (src_mpi/Particle/ComputeAcceleration.cpp:
 * 14-190) and calculateTimeStepIrr (src_mpi/Particle/UpdateParticle.cpp:
 * 151-241).  A step equals the host integrator's step bit for bit (the same
 * FP64 operations in the same order); the level rule's logarithm is the one
 * place where the device and the host libm could differ, and level decisions
 * within 1e-12 of a power-of-two boundary are counted (borderline).
 */
#ifndef ABYSS_IRR_H
#define ABYSS_IRR_H
#ifdef __cplusplus
extern "C" {
#endif

struct abyss_ac;

/* Run this integration's irregular levels on the GPU of its context (on != 0)
 * or on the host threads (on == 0, the default).  Results are the same either
 * way.  Not while a split block is open.  The device keeps a copy of the state;
 * before each block's levels the particles the host committed since (the last
 * regular block's targets) are sent up, and afterwards every particle's
 * irregular fields come back. */
int abyss_ac_set_device_irregular(struct abyss_ac *ac, int on);
/* Whether the device path is on, how many level decisions were borderline, the
 * wall seconds spent packing and copying state for it, and (cycles6, may be
 * NULL) the SM clock cycles one block spent in each part of the levels, summed:
 * member list, (unused), steps, barrier, commit and next level, barrier. */
int abyss_ac_device_irregular_info(const struct abyss_ac *ac, int *on, long long *borderline,
                                   double *sec_copy, long long *cycles6);

/* Whole blocks on the GPU (on != 0): the state of record moves to the device
 * and a block never leaves it -- the next block's particles
 * (updateNextRegTime, src_mpi/RootRoutines.cpp:1310-1338), the irregular
 * levels above, the regular force, the corrector and commit
 * (updateRegularParticleCuda and RegCudaUpdate, ComputeAcceleration.cpp:
 * 405-661, WorkerRoutines.cpp:124-143), the regular and irregular time steps
 * and the neighbour radius (UpdateParticle.cpp:108-139, 151-241, 314-407).
 * The host learns each block's time and size only.  Results equal the host
 * integrator's bit for bit, as above; level decisions within 1e-12 of a
 * power-of-two boundary are counted.  The particles are read back when the
 * state is asked for (abyss_ac_get_state, abyss_ac_energy, abyss_ac_save,
 * abyss_ac_write_snapshot, and on == 0); abyss_ac_last_regular gives the last
 * device block.  The split form (abyss_ac_begin_block) is refused while on.
 * Not while a split block is open. */
int abyss_ac_set_device_resident(struct abyss_ac *ac, int on);
/* Whether whole blocks run on the device, the borderline level decisions of
 * their regular steps, and the wall seconds spent copying the whole state
 * between host and device. */
int abyss_ac_device_resident_info(const struct abyss_ac *ac, int *on, long long *borderline, double *sec_sync);

/* One irregular step of each of `count` particles idx[k] of an n-particle
 * state, on GPU `device`, nothing committed: the arguments of
 * abyss_host_irregular_steps (include/abyss_host.h) plus the level inputs of
 * calculateTimeStepIrr -- time_block (block times are multiples of
 * 2^time_block, -62 <= time_block <= -1), eta_irr, and per particle lv_reg,
 * cur_reg and tb_reg -- and its outputs lv_irr, dt_irr, tb_irr (any of the
 * three may be NULL).  t_irr and dt_irr must lie on the 2^time_block grid. */
int abyss_device_irregular_steps(int device, int n, const double *x, const double *v, const double *mass,
                                 const double *a_tot, const double *a_reg, const double *a_irr,
                                 const double *t_reg, const double *t_irr, const double *dt_irr,
                                 const int *nnb, const int *nb, int nb_stride, double eps2, double scale,
                                 int time_block, double eta_irr, const int *lv_reg,
                                 const unsigned long long *cur_reg, const unsigned long long *tb_reg, int count,
                                 const int *idx, double *new_pos, double *new_vel, double *a_irr_out,
                                 double *a_tot_out, int *lv_irr_out, double *dt_irr_out,
                                 unsigned long long *tb_irr_out);

#ifdef __cplusplus
}
#endif
#endif
