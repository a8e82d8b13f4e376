/* abyss_ac.h -- C ABI of the host Ahmad-Cohen integrator (libabyss_reg.so).
 *
 * The host keeps the reference's 4th-order Hermite predictor/corrector, block
 * timesteps and regular/irregular scheduling (src_mpi/RootRoutines.cpp:240-330,
 * 448-1075, 1310-1338; src_mpi/WorkerRoutines.cpp:46-143;
 * the src_mpi/Particle/ sources) and calls the GPU regular force through abyss_reg.h
 * at every regular block, in place of calculateRegAccelerationOnGPU
 * (src_mpi/cuda/CalculateRegularAcceleration.cpp:27-324).
 *
 * Units: N-body (G = 1).  Code time runs over [0, 1] and one code-time unit is
 * t_end N-body time units (the reference's EnzoTimeStep, DefaultGlobal.cpp:92).
 * Irregular steps and the corrector run on host threads; every phase computes
 * all of a block's new values before committing any of them, so results do not
 * depend on thread scheduling.
 */
#ifndef ABYSS_AC_H
#define ABYSS_AC_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct abyss_ac abyss_ac;
struct abyss_ctx;

typedef struct abyss_ac_params {
  double eps2;     /* softening^2, force terms only */
  double eta_reg;  /* Aarseth accuracy parameter, regular steps (reference: eta, def.h:36) */
  double eta_irr;  /* Aarseth accuracy parameter, irregular steps */
  int fix_nb;      /* target neighbour count (FixNumNeighbor, def.h:18) */
  int nb_max;      /* radius-adaptation scale and list capacity (NumNeighborMax, def.h:20) */
  double t_end;    /* N-body time of code time 1 */
  int threads;     /* host threads (0 = all) */
} abyss_ac_params;

typedef struct abyss_ac_stats {
  long long blocks;        /* regular blocks advanced */
  long long reg_steps;     /* particle regular steps */
  long long irr_steps;     /* particle irregular steps */
  long long irr_levels;    /* irregular block levels processed */
  long long radius_retries;/* regular calls re-run after a list overflow */
  double pairs;            /* regular-force pairs (m * N summed) */
  double sec_reg_gpu;      /* wall seconds in the regular-force ABI calls */
  double sec_reg_host;     /* wall seconds in the host regular corrector/update */
  double sec_irr;          /* wall seconds in irregular steps */
  double sec_init;         /* wall seconds in initialisation */
} abyss_ac_stats;

/* ctx must outlive the integrator.  r2nb = initial squared neighbour radii. */
int abyss_ac_create(struct abyss_ctx *ctx, const abyss_ac_params *p, int n, const double *x,
                    const double *v, const double *mass, const double *r2nb, abyss_ac **out);
int abyss_ac_destroy(abyss_ac *ac);
/* Advance through the next regular block (its irregular levels first, then the
 * regular step).  *done = 1 once code time 1 is reached. */
int abyss_ac_advance_block(abyss_ac *ac, int *done);
/* Split form of abyss_ac_advance_block, for callers that batch the regular
 * force of many integrators into one launch (abyss_ens.h):
 *   begin_block   runs the irregular levels up to the next regular block and
 *                 opens it: m targets at new_time (code time), time_scale;
 *   block_targets the block's targets [m] (ascending particle index);
 *   block_state   the un-predicted state to upload for the force: x, v, a0, a1
 *                 [n][3], t0, mass, r2nb [n];
 *   end_block     hands over the regular force of the targets (rows in target
 *                 order, as abyss_fetch returns them) and commits the block.
 * When a target's list did not fit in list_cap, end_block shrinks that
 * target's radius, commits nothing and returns ABYSS_WARN_OVERFLOW: fetch the
 * state again, redo the force and call end_block again. */
int abyss_ac_begin_block(abyss_ac *ac, int *m, double *new_time, double *time_scale, int *done);
int abyss_ac_block_targets(const abyss_ac *ac, int *targets);
int abyss_ac_block_state(const abyss_ac *ac, double *x, double *v, double *a0, double *a1, double *t0,
                         double *mass, double *r2nb);
int abyss_ac_end_block(abyss_ac *ac, const double *acc, const double *jerk, const double *acc_irr,
                       const double *jerk_irr, const int *nnb, const int *list, int list_cap, int *done);

/* Serving loop over k integrations whose regular forces share the ensemble e
 * (include/abyss_ens.h); integration i owns cluster slots[i] and must have
 * been created with threads = 1.  `threads` host workers advance the
 * integrations independently, block by block: a worker runs an integration's
 * irregular levels up to its next regular block, writes the block's state into
 * the ensemble's pinned staging and queues it; the calling thread runs every
 * queued block as one ensemble wave (mode ABYSS_ENS_BATCHED or _GRAPH), one wave
 * at a time, back to back, and hands each block's rows back to a worker, which
 * applies the corrector and opens the next block at once.  No integration waits
 * for another's host work, and each one's results do not depend on which
 * blocks shared its waves.
 * The call returns once stop_after integrations (0 = all) have reached code
 * time 1, or after the wave that ends past budget_ms of wall time (<= 0: no
 * budget); blocks in flight are committed first, and an integration whose
 * block was queued but not run keeps it open for the next call.
 * status[i]: one of the codes below, or a negative ABYSS_ERR_* code;
 * blocks[i]: regular blocks it committed in this call.  *gpu_ms: GPU time of
 * the waves, *waves: their count, *stats: where the time went (any of the three
 * may be NULL). */
#define ABYSS_ROUND_ADVANCED 0       /* between blocks, or a block open */
#define ABYSS_ROUND_ADVANCED_DONE 1  /* its last block was committed: code time 1 reached */
#define ABYSS_ROUND_FINISHED 2       /* nothing to do: code time 1 had been reached */
#define ABYSS_ROUND_REDO 3           /* a list overflowed: radii shrunk, the block runs again */
struct abyss_ens;
typedef struct abyss_serve_stats {
  double wall_s;      /* the whole call */
  double prep_s;      /* dispatcher: staged upload, wave set-up, launch */
  double wait_s;      /* dispatcher: waiting for a wave's results */
  double hand_s;      /* dispatcher: handing rows back to the workers */
  double idle_s;      /* dispatcher: no block queued */
  double worker_s;    /* host workers: busy time, summed over workers */
  long long rows;     /* targets over all waves */
} abyss_serve_stats;
int abyss_ac_serve_run(struct abyss_ens *e, int k, abyss_ac *const *acs, const int *slots, double eps2,
                       int mode, int threads, double budget_ms, int stop_after, int *status, int *blocks,
                       float *gpu_ms, int *waves, abyss_serve_stats *stats);

/* Advance until code time >= t_code (<= 1). */
int abyss_ac_run(abyss_ac *ac, double t_code);
/* Current code time (the last regular block time reached). */
double abyss_ac_time(const abyss_ac *ac);
/* Positions/velocities [n][3], neighbour counts, squared radii (any may be NULL). */
int abyss_ac_get_state(const abyss_ac *ac, double *x, double *v, int *nnb, double *r2nb);
/* Total energy (FP64, softened) of the current state; valid when all particles
 * share one time (start, end). */
int abyss_ac_energy(abyss_ac *ac, double *energy);
int abyss_ac_get_stats(const abyss_ac *ac, abyss_ac_stats *st);
/* The last regular call: m targets, the predicted j-set (n x 3 FP64), the
 * squared radii used and the GPU results, for parity checks. */
int abyss_ac_last_regular(const abyss_ac *ac, int *m, int *targets, double *px, double *pv,
                          double *r2nb, double *acc_reg, double *jerk_reg, int *nnb, int *list,
                          int list_cap);
const char *abyss_ac_last_error(const abyss_ac *ac);
/* Wall seconds outside the stats' timers, summed over the run: [0] filling,
 * uploading and predicting the j-set of each regular block, [1] finding each
 * next regular block (updateNextRegTime, RootRoutines.cpp:1310-1338). */
int abyss_ac_host_timers(const abyss_ac *ac, double *sec2);
/* Particle count and parameters of an integration (either may be NULL). */
int abyss_ac_info(const abyss_ac *ac, int *n, abyss_ac_params *p);

#ifdef __cplusplus
}
#endif
#endif
