// Irregular steps on the device: the Ahmad-Cohen irregular force of every
// particle due before the next regular block, level by level, with the level
// loop itself on the GPU (irregular.cu).  Host-side interface, used by the host
// integrator (host/ac_integrator.cpp) and the C ABI (include/abyss_irr.h).
//
// Reference: the IrrForce/IrrUpdate tasks (src_mpi/WorkerRoutines.cpp:46-64,
// 76-87) dispatched level by level from the skip list of
// src_mpi/RootRoutines.cpp:488-1005; per particle computeAccelerationIrr
// (src_mpi/Particle/ComputeAcceleration.cpp:14-190) and calculateTimeStepIrr
// (src_mpi/Particle/UpdateParticle.cpp:151-241).
#pragma once
#include <cstdint>
#include <string>

namespace abyss_irr {

typedef unsigned long long ULL;

// One particle's state as the irregular phase reads and writes it (the host
// integrator's fields of record, packed for one copy each way).
struct Image {
  double x[3], v[3], m, t_irr, t_reg, dt_irr;
  double a_tot[12], a_reg[12], a_irr[12];  // [d][k] row-major, 3 x 4
  ULL cur_irr, tb_irr, next_irr, new_cur_irr, cur_reg, tb_reg;
  double r2nb, dt_reg;  // read by whole regular blocks on the device only
  int lv_irr, lv_reg, nnb, index;
  long long list_off;  // first of its nnb neighbours in the staged lists
};

// The fields an irregular phase changes, per particle, as they come back.
struct Changed {
  double x[3], v[3], t_irr, dt_irr;
  double a_tot[12], a_irr[12];
  ULL cur_irr, tb_irr, next_irr, new_cur_irr;
  int lv_irr, touched;  // touched: stepped since the last download
};

// Constants of one integration's irregular phase.
struct Params {
  double scale;      // EnzoTimeStep (N-body time of code time 1)
  double time_step;  // 2^time_block
  double eps2;       // softening^2 of the force terms
  double eta_irr;    // Aarseth accuracy parameter of irregular steps
  double ln2;        // log(2.0) as the host's libm gives it (the level rule's divisor)
  int time_block;
  ULL next_reg_block;  // levels up to this block time are run
};

// What a run of the level loop did.
struct RunStats {
  long long levels = 0, steps = 0;
  // level decisions whose log(dt)/log(2) lay within 1e-12 of an integer: the
  // only place where the device's log and the host's libm log could pick
  // different levels (counted, so that a run can show it met none)
  long long borderline = 0;
  // SM clock cycles of one block in each part of a level, summed: member
  // list, (unused), steps, barrier, commit and next level, barrier
  long long cycles[6] = {0, 0, 0, 0, 0, 0};
};

// Constants of whole regular blocks on the device (engine_next_block ..
// engine_correct_block): the irregular phase's plus the regular step's rules.
struct BlockParams {
  Params irr;        // next_reg_block: the block being corrected
  double eta_reg;    // Aarseth accuracy parameter of regular steps
  ULL block_max;     // block count of code time 1
  int fix_nb;        // FixNumNeighbor of updateRadius
  int nb_max;        // NumNeighborMax of updateRadius (also the list capacity)
};

// Device arrays of a regular-force context's j-set state (context.cu), which
// engine_fill_jset writes: x, v, a0, a1 [n][3], t0, mass, r2nb [n].
struct JsetDst {
  double *x, *v, *a0, *a1, *t0, *mass, *r2nb;
};

// Device results of the context's last regular-force launch, row k being the
// block's k-th target: acc/jerk regular and irregular [m][3], nnb [m], list
// [m][cap] ascending.
struct RegResults {
  const double *acc_reg, *jerk_reg, *acc_irr, *jerk_irr;
  const int *nnb, *list;
  int cap;
};

struct Engine;

// Engine on `device` (the context's device); ABYSS_* codes.
int engine_create(int device, Engine **out);
void engine_destroy(Engine *e);
const char *engine_error(const Engine *e);
// How the engine's calls wait for the GPU: spin_us < 0 (the default) the
// stream synchronisation; else poll for spin_us microseconds, then sleep in a
// blocking event wait (abyss_set_wait of include/abyss_reg.h).
int engine_set_wait(Engine *e, int spin_us);
// Size the device state for n particles with lists of capacity cap (keeps
// the state when the sizes are unchanged; a smaller n with the same capacity
// reuses the arrays, cleared).
int engine_reserve(Engine *e, int n, int cap);
// Engines kept for reuse between integrations (an engine's arrays and pinned
// staging are allocated once for the largest cluster it held; allocating them
// per integration would synchronize the device under every other stream).
// engine_take gives a pooled engine of `device` or a new one; engine_give
// returns one to the pool (or frees it when the pool is full).
int engine_take(int device, Engine **out);
void engine_give(Engine *e);
// Pinned staging: n images and n x cap list entries (packed: image k's list
// starts at its list_off).
Image *engine_images(Engine *e);
int *engine_lists(Engine *e);
// Scatter the first `count` staged images (each carrying its particle index)
// and their lists (list_entries in all) into the device state.
int engine_upload(Engine *e, int count, long long list_entries);
// The level loop up to p.next_reg_block on the device state, on `stream` (a
// cudaStream_t; null: the engine's own).  Returns ABYSS_OK, ABYSS_ERR_STATE (a
// time step out of range: nothing of that level committed), ABYSS_ERR_TIMEOUT
// or ABYSS_ERR_CUDA.
int engine_run_levels(Engine *e, const Params &p, RunStats *st, void *stream = nullptr);
// Copy the changed fields of every particle into the pinned staging
// (engine_changed()[i] is particle i, its `touched` flag set when a run since
// the last download stepped it) and clear the flags.
int engine_download(Engine *e);
Changed *engine_changed(Engine *e);
// One step of each listed particle from the device state, nothing committed:
// new position and velocity, a_irr and a_tot [3][4], and the new level, step
// and block count of calculateTimeStepIrr.
int engine_steps(Engine *e, const Params &p, int count, const int *idx, double *new_pos, double *new_vel,
                 double *a_irr, double *a_tot, int *lv_irr, double *dt_irr, ULL *tb_irr);

// ---- whole regular blocks with the state resident on the device
// (src_mpi/RootRoutines.cpp:1310-1338 updateNextRegTime and the regular half
// of the block loop; UpdateParticle.cpp:108-139, 314-407;
// ComputeAcceleration.cpp:405-661).  All of them run on `stream` (the
// regular-force context's), after the engine holds the whole state
// (engine_upload of every particle).
//
// The next regular block: tmin = the smallest cur_reg + tb_reg not above
// block_max (block_max when there is none) and its m particles, in ascending
// index (engine_block_targets, device memory).  Synchronizes.
int engine_next_block(Engine *e, void *stream, ULL block_max, ULL *tmin, int *m);
const int *engine_block_targets(const Engine *e);
// The context's j-set state from the engine's: t0 is t_reg for a particle
// without neighbours, else t_irr (CalculateRegularAcceleration.cpp:371-374).
int engine_fill_jset(Engine *e, void *stream, const JsetDst &d);
// r2nb *= 0.8 for every target k whose list overflowed (nnb[k] > cap).
int engine_shrink_radii(Engine *e, void *stream, int m, const int *nnb, int cap);
// Corrector and commit of the block's m targets from the context's results
// (updateRegularParticleCuda, RegCudaUpdate, calculateTimeStepReg/Irr,
// updateRadius), every target from the pre-block state.  Synchronizes.
// Returns ABYSS_OK, ABYSS_ERR_STATE (a time step out of range; the block is
// committed, as on the host) or ABYSS_ERR_CUDA; borderline level decisions
// are added to *borderline.
int engine_correct_block(Engine *e, void *stream, const BlockParams &bp, int m, const RegResults &r,
                         long long *borderline);
// Every particle's fields into the pinned staging: engine_images()[i] is
// particle i (list_off = i * cap), its list at engine_lists() + i * cap.
int engine_download_all(Engine *e);

}  // namespace abyss_irr
