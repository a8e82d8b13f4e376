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

struct Engine;

// Engine on `device` (the context's device); ABYSS_* codes.
int engine_create(int device, Engine **out);
void engine_destroy(Engine *e);
const char *engine_error(const Engine *e);
// Size the device state for n particles with lists of capacity cap (keeps
// the state when the sizes are unchanged).
int engine_reserve(Engine *e, int n, int cap);
// Pinned staging: n images and n x cap list entries (packed: image k's list
// starts at its list_off).
Image *engine_images(Engine *e);
int *engine_lists(Engine *e);
// Scatter the first `count` staged images (each carrying its particle index)
// and their lists (list_entries in all) into the device state.
int engine_upload(Engine *e, int count, long long list_entries);
// The level loop up to p.next_reg_block on the device state.  Returns
// ABYSS_OK, ABYSS_ERR_STATE (a time step out of range: nothing of that level
// committed), ABYSS_ERR_TIMEOUT or ABYSS_ERR_CUDA.
int engine_run_levels(Engine *e, const Params &p, RunStats *st);
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

}  // namespace abyss_irr
