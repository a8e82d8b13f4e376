/* abyss_reg.h -- C ABI of the B200 Ahmad-Cohen regular-force library
 * (libabyss_reg.so).  Plain pointers and sizes only.
 *
 * Two layers:
 *   1. The reference-compatible drop-in (abyss_reg_compat.h): the six
 *      entry points of src_mpi/cuda/cuda_functions.h:3-10.
 *   2. This status-returning context API, used by the drop-in, the host
 *      integrator, the batched ensemble and the serving loop.
 *
 * Conventions
 *   - Every function returns ABYSS_OK (0) or a negative ABYSS_ERR_* code;
 *     abyss_last_error() gives a message.  Nothing traps the GPU: a list
 *     longer than its capacity is reported (ABYSS_WARN_OVERFLOW, exact
 *     counts, truncated lists), never asserted.
 *   - Vectors are row-major double [k][3]; lists are int [m][list_cap],
 *     ascending particle index, row r holding target r's neighbours.
 *   - A "j-set" is the n particles of one cluster; "targets" are the m
 *     active particle indices of a regular block (0 <= target < n).
 *   - Neighbour rule (src_mpi/Particle/ComputeAcceleration.cpp:285): j != i is
 *     a neighbour of target i when |x_j - x_i|^2 < r2nb[i] in FP64; its force
 *     goes to the irregular part, every other j's to the regular part.
 *     Softening eps2 enters the force terms only.
 *   - One context per host thread at a time; calls on one context are
 *     ordered on the context's CUDA stream.
 */
#ifndef ABYSS_REG_H
#define ABYSS_REG_H
#ifdef __cplusplus
extern "C" {
#endif

#define ABYSS_OK 0
#define ABYSS_WARN_OVERFLOW 1   /* some target had more neighbours than list_cap */
#define ABYSS_ERR_ARG (-1)      /* bad argument (size, index, pointer) */
#define ABYSS_ERR_CUDA (-2)     /* CUDA runtime error */
#define ABYSS_ERR_OOM (-3)      /* device or pinned allocation failed */
#define ABYSS_ERR_TIMEOUT (-4)  /* a bounded device wait ran out */
#define ABYSS_ERR_STATE (-5)    /* call out of order (e.g. no j-set uploaded) */
#define ABYSS_ERR_NODEVICE (-6) /* no usable CUDA device */

typedef struct abyss_ctx abyss_ctx;

/* Launch shape.  Zero fields are chosen by the library (or by a tuning table
 * installed with abyss_set_tuning_table). */
typedef struct abyss_tuning {
  int kernel;  /* 1 = tile kernel (i in registers, j-tiles by TMA), 2 = j-major kernel,
                  3 = tile kernel with packed FP32x2 pair arithmetic,
                  4 = tile kernel whose 4 warps share 32 x ipt targets (ipt 1 or 2) and
                      split each j-tile, for small active sets (double-single),
                  5 = kernel 4 with packed FP32x2 pair arithmetic (over a thread's two
                      targets for ipt 2, over two j for ipt 1) */
  int mode;    /* tile kernel: 1 = anchor offsets on spatially ordered targets, 2 = double-single */
  int threads; /* tile kernel: 128 or 256 */
  int ipt;     /* tile: targets per thread 1, 2, 4;  j-major: targets per pass 1, 2, 4, 8 */
  int j_split; /* j-chunks per target (0 = auto) */
  int grid;    /* tile kernel persistent grid size (0 = auto) */
  int unroll;  /* tile kernel: j per warp vote, 1 or 2 (0 = first available) */
  int min_blocks; /* tile kernel: register cap as resident CTAs per SM (0 = first available) */
} abyss_tuning;

/* Number of compiled tile-kernel shapes and the shape of entry i as
 * (threads, ipt, anchor, packed, unroll, min_blocks); kernel = 3 when packed. */
int abyss_tile_variants(void);
int abyss_tile_variant(int i, int *shape6);

/* Replaces the reference's _InitializeDevice/_OpenDevice state
 * (src_mpi/cuda/cuda_my_acceleration.cu:782-882, 886-903) with an explicit
 * context on `device`. */
int abyss_create(int device, abyss_ctx **out);
/* Frees every device and pinned buffer (the reference's CloseDevice frees
 * nothing, cuda_my_acceleration.cu:905-947). */
int abyss_destroy(abyss_ctx *ctx);
const char *abyss_last_error(const abyss_ctx *ctx);
/* Opaque cudaStream_t of the context (all work of the context runs on it). */
void *abyss_stream(abyss_ctx *ctx);
int abyss_synchronize(abyss_ctx *ctx);
/* How the context's calls wait for the GPU.  spin_us < 0 (the default): the
 * stream synchronisation, whose thread keeps its core while it waits.
 * spin_us >= 0: poll for at most spin_us microseconds, then sleep in a blocking
 * event wait, so that a thread whose call waits behind other work on a busy GPU
 * leaves its core to other host threads (many contexts driven from more host
 * threads than cores).  Results do not depend on it.  No reference counterpart:
 * the reference waits in cudaStreamSynchronize (cuda_my_acceleration.cu:242). */
int abyss_set_wait(abyss_ctx *ctx, int spin_us);

/* Pre-size buffers for n particles, m targets, list capacity list_cap
 * (replaces the grow-on-demand reallocation at cuda_my_acceleration.cu:635-727). */
int abyss_reserve(abyss_ctx *ctx, int n, int m, int list_cap);

/* Upload un-predicted FP64 state (host arrays); prediction then runs on the
 * device.  x, v, a0 (= a_tot[.][0]), a1 (= a_tot[.][1]) are [n][3]; t0 is the
 * time each particle was last advanced to (CurrentTimeReg when it has no
 * neighbours, else CurrentTimeIrr: CalculateRegularAcceleration.cpp:371-374). */
int abyss_upload_state(abyss_ctx *ctx, int n, const double *x, const double *v,
                       const double *a0, const double *a1, const double *t0,
                       const double *mass, const double *r2nb);
/* Second-order prediction of the whole j-set to new_time on the device
 * (UpdateParticle.cpp:37-59): dt = (new_time - t0) * time_scale. */
int abyss_predict(abyss_ctx *ctx, double new_time, double time_scale);
/* Upload an already predicted j-set (positions/velocities [n][3]). */
int abyss_upload_predicted(abyss_ctx *ctx, int n, const double *px, const double *pv,
                           const double *mass, const double *r2nb);

/* Copy the predicted j-set back: px, pv [n][3] FP64, vm [n][4] FP32
 * (vx, vy, vz, m) as the force kernels read it; any pointer may be NULL. */
int abyss_read_predicted(abyss_ctx *ctx, double *px, double *pv, float *vm);

/* Copy the m target indices to the device. */
int abyss_set_targets(abyss_ctx *ctx, int m, const int *targets);
/* Enqueue the regular force of the current targets on the context stream
 * (asynchronous).  tuning may be NULL. */
int abyss_launch(abyss_ctx *ctx, double eps2, int list_cap, const abyss_tuning *tuning);
/* Wait for the last launch and copy its results to host memory; any output
 * pointer may be NULL.  acc/jerk are [m][3]; nnb [m] holds exact counts; list is
 * [m][list_cap].  Returns ABYSS_WARN_OVERFLOW (with *overflow_rows set) when a
 * list was truncated. */
int abyss_fetch(abyss_ctx *ctx, double *acc_reg, double *jerk_reg, double *acc_irr,
                double *jerk_irr, int *nnb, int *list, int *overflow_rows);
/* set_targets + launch + fetch. */
int abyss_regular_force(abyss_ctx *ctx, int m, const int *targets, double eps2, int list_cap,
                        const abyss_tuning *tuning, double *acc_reg, double *jerk_reg,
                        double *acc_irr, double *jerk_irr, int *nnb, int *list,
                        int *overflow_rows);

/* The shape the last abyss_launch used (after auto selection) and its j-chunk count. */
int abyss_last_plan(const abyss_ctx *ctx, abyss_tuning *plan, int *n_chunks);
/* The order in which the last launch processed its targets: rows[s] is the
 * target row (index into the targets of abyss_set_targets) in processing slot
 * s, m entries.  Consecutive slots share an i-block of threads x ipt targets;
 * in anchor mode the slots follow the targets' Hilbert-curve order and each
 * i-block's offsets are taken from the centre of its targets' bounding box.
 * Identity otherwise.
 * Synchronizes the stream.  No reference counterpart (diagnostics). */
int abyss_last_order(abyss_ctx *ctx, int *rows);
/* Time subsequent launches with CUDA events on the context stream: on == 1
 * each phase, on == 2 the whole launch with two events (the events between
 * phases take a few microseconds of the stream themselves), 0 off. */
int abyss_set_profiling(abyss_ctx *ctx, int on);
/* Milliseconds of the last profiled launch: [0] target ordering, [1] force
 * kernel, [2] finalize; with on == 2, [1] is the whole launch and [0] = [2] = 0.
 * Synchronizes the stream. */
int abyss_last_timing(abyss_ctx *ctx, float *ms3);
/* Auto-selection table from the autotuner: k entries, each (m_max, tuning);
 * the first entry with m <= m_max wins.  k = 0 restores the built-in rule. */
int abyss_set_tuning_table(abyss_ctx *ctx, int k, const int *m_max, const abyss_tuning *entries);

/* Regular force for callers that cannot allocate device memory (no counterpart
 * in the reference).  For hosts whose GPU memory is owned by another allocator,
 * held to a hard budget, or on a path where cudaMalloc/cudaFree may not run:
 * the caller passes device buffers for inputs (predicted j-set px, py, pz,
 * pvx, pvy, pvz, mass, r2nb [n]; vm [n][4] = (vx, vy, vz, m) as float; targets
 * [m]) and outputs (acc/jerk [m][3], nnb [m], list [m][list_cap]); every
 * intermediate buffer is a fixed array inside the library and nothing is
 * allocated.  Limits: m <= 4096, list_cap <= 256; larger sizes are rejected
 * with ABYSS_ERR_ARG and a message on stderr.  px, py, pz, vm must be 16-byte
 * aligned.  The array is shared by all calls on a device and keeps the last
 * call's contents; calls that overlap on the GPU race on it and must be
 * serialized by the caller.  Work runs on `stream` (a cudaStream_t, may be 0)
 * and the call returns when it has finished.  The first call on a device sets
 * the array up.  Returns ABYSS_OK, ABYSS_WARN_OVERFLOW or an ABYSS_ERR_* code. */
int abyss_regular_force_noalloc(int n, const double *px, const double *py, const double *pz,
                                const float *vm, const double *pvx, const double *pvy,
                                const double *pvz, const double *mass, const double *r2nb, int m,
                                const int *targets, double eps2, int list_cap, double *acc_reg,
                                double *jerk_reg, double *acc_irr, double *jerk_irr, int *nnb,
                                int *list, void *stream);

/* Second and third time derivatives of the acceleration of n particles at one
 * common time: the initialisation pass of the scheme (the reference's
 * CalculateAcceleration23, src_mpi/Particle/Initialize.cpp:102-185, run there
 * on the host for every particle).  Split into regular (r^2 >= R^2, unsoftened
 * r^2) and irregular parts; eps2 is added to r^2 in the force terms.  FP64 on
 * the device, one target per thread summing j in ascending order in the
 * reference's operation order, so each value equals that sequential loop bit
 * for bit.  Host arrays: x, v, a0 (acceleration), a1 (jerk) [n][3], mass and
 * r2nb [n]; outputs [n][3].  Synchronous. */
int abyss_init_derivs23(abyss_ctx *ctx, int n, const double *x, const double *v, const double *mass,
                        const double *r2nb, const double *a0, const double *a1, double eps2,
                        double *reg2, double *reg3, double *irr2, double *irr3);

/* FP64 total energy (kinetic + softened potential) of n particles. */
int abyss_energy(abyss_ctx *ctx, int n, const double *x, const double *v, const double *mass,
                 double eps2, double *energy);

#ifdef __cplusplus
}
#endif
#endif
