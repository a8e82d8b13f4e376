/* abyss_ens.h -- batched regular force over many independent clusters
 * (libabyss_reg.so).
 *
 * The reference integrates one cluster per run and calls its GPU regular force
 * once per regular block (src_mpi/RootRoutines.cpp:1026-1075).  An ensemble
 * holds K clusters of uneven size resident on one GPU; a "wave" is one regular
 * block of any subset of them (each cluster with its own time and its own
 * active set).  A wave runs as one device prediction, ONE persistent launch of
 * the tile kernel over a work list of (cluster, target block, j-chunk) items and
 * one finalize pass; with ABYSS_ENS_GRAPH those three are replayed from a CUDA
 * graph captured once.  ABYSS_ENS_PLAIN runs the same kernels one cluster per
 * launch, the baseline the batched form is measured against.
 *
 * Indices are cluster-local (0 <= target < n_k), as are the returned lists.
 * Rows of the outputs follow the order of the wave's clusters and targets.
 */
#ifndef ABYSS_ENS_H
#define ABYSS_ENS_H
#ifdef __cplusplus
extern "C" {
#endif

struct abyss_ctx;
struct abyss_tuning;
typedef struct abyss_ens abyss_ens;

#define ABYSS_ENS_BATCHED 0  /* one launch per wave */
#define ABYSS_ENS_GRAPH 1    /* the batched wave replayed from a captured CUDA graph */
#define ABYSS_ENS_PLAIN 2    /* one launch per cluster (baseline) */

/* n_clusters clusters of n_per_cluster[k] particles; list_cap = neighbour-list
 * capacity per target.  Device memory for every particle being a target is
 * reserved up front (state, outputs and work buffers), so waves never allocate. */
int abyss_ens_create(struct abyss_ctx *ctx, int n_clusters, const int *n_per_cluster, int list_cap,
                     abyss_ens **out);
int abyss_ens_destroy(abyss_ens *e);
/* An empty ensemble with room for `capacity` particles in at most max_clusters
 * clusters (all device memory reserved here).  Clusters then come and go: */
int abyss_ens_create_arena(struct abyss_ctx *ctx, int capacity, int max_clusters, int list_cap,
                           abyss_ens **out);
/* Place a cluster of n particles (first fit, 32-particle aligned); *k is its id.
 * ABYSS_ERR_OOM when no slot or no contiguous room is free (admission refused). */
int abyss_ens_attach(abyss_ens *e, int n, int *k);
/* Release cluster k's slot and particle range. */
int abyss_ens_detach(abyss_ens *e, int k);
/* Largest contiguous free particle range. */
int abyss_ens_free_particles(const abyss_ens *e);
/* j-particles per chunk of the work list (>= 128; default 2048): cluster k is
 * split into min(16, ceil(n_k / j_per_chunk)) j-chunks in every wave.  Small
 * chunks spread a wave of small clusters over more of the GPU (lower latency
 * per wave); the split depends on n_k alone, so results stay the same alone
 * and in any mix.  Results change with this setting at the FP32 rounding level. */
int abyss_ens_set_chunk(abyss_ens *e, int j_per_chunk);
/* Neighbour-list capacity per target (the row stride of fetched lists). */
int abyss_ens_list_cap(const abyss_ens *e);
/* Launch shape of the ensemble's force kernel and its j-chunk length by
 * cluster size, as an autotuner picked them (abyss_b200/autotune.py
 * tune_ensemble).  shape: a compiled tile shape with double-single offsets
 * (kernel 1 or 3, mode 2, at least 128 targets per block), NULL to keep the
 * shape; k entries (n_max, j_per_chunk) in rising n_max: the first entry with
 * n_k <= n_max sets the chunk length of a cluster of n_k particles, larger
 * clusters take abyss_ens_set_chunk's.  Applies from the next wave.  A
 * cluster's chunking depends on its own size only, so its results stay the
 * same alone and in any mix.  No reference counterpart: the reference fixes
 * BatchSize 64, GridDimY 64 and NNB_per_block 128 at compile time
 * (src_mpi/def.h:77-79). */
int abyss_ens_set_tuning(abyss_ens *e, const struct abyss_tuning *shape, int k, const int *n_max,
                         const int *j_per_chunk);
/* The launch shape in use. */
int abyss_ens_get_shape(const abyss_ens *e, struct abyss_tuning *shape);
/* Device bytes the ensemble holds (for admission control). */
long long abyss_ens_device_bytes(const abyss_ens *e);
/* Un-predicted FP64 state of cluster k, as abyss_upload_state. */
int abyss_ens_upload_state(abyss_ens *e, int k, const double *x, const double *v, const double *a0,
                           const double *a1, const double *t0, const double *mass,
                           const double *r2nb);
/* Staged upload, for callers that refresh many clusters per wave: after
 * abyss_ens_stage_reserve (pinned host memory for the whole arena, 120 B per
 * particle of capacity), abyss_ens_stage gives cluster k's seven state arrays
 * inside it (same layout as abyss_ens_upload_state; the caller writes them, from
 * any thread), and abyss_ens_upload_staged queues the copies of the listed
 * clusters on the ensemble's stream, merged into one copy per array for each
 * run of listed clusters that are adjacent in the arena.  Clusters not listed
 * are not written.  The staged memory must not change until the next wave has
 * been launched and fetched. */
int abyss_ens_stage_reserve(abyss_ens *e);
int abyss_ens_stage(abyss_ens *e, int k, double **x, double **v, double **a0, double **a1, double **t0,
                    double **mass, double **r2nb);
int abyss_ens_upload_staged(abyss_ens *e, int nk, const int *clusters);
/* Define the next wave: nk clusters, each predicted to new_time[i] with
 * time_scale[i] and m_per[i] targets (concatenated in targets_local). */
int abyss_ens_set_wave(abyss_ens *e, int nk, const int *clusters, const double *new_time,
                       const double *time_scale, const int *m_per, const int *targets_local);
/* Run the wave (mode = ABYSS_ENS_BATCHED, _GRAPH or _PLAIN); asynchronous. */
int abyss_ens_launch(abyss_ens *e, double eps2, int mode, const struct abyss_tuning *tuning);
/* Wait and copy the wave's results (rows in wave order); any pointer may be NULL. */
int abyss_ens_fetch(abyss_ens *e, double *acc_reg, double *jerk_reg, double *acc_irr,
                    double *jerk_irr, int *nnb, int *list, int *overflow_rows);
/* As abyss_ens_fetch, without copies into caller memory: the results land in
 * pinned host memory owned by the ensemble and the pointers returned stay valid
 * until the next abyss_ens_fetch_view or abyss_ens_destroy. */
int abyss_ens_fetch_view(abyss_ens *e, const double **acc_reg, const double **jerk_reg, const double **acc_irr,
                         const double **jerk_irr, const int **nnb, const int **list, int *overflow_rows);
/* Two waves in flight.  abyss_ens_submit uploads the listed clusters' staged
 * state, describes the wave, launches it (mode ABYSS_ENS_BATCHED or _GRAPH) and
 * queues the copies of its results, all asynchronously, and returns a ticket;
 * abyss_ens_collect(ticket) waits for that wave and returns its rows (in wave
 * order) in pinned memory that stays valid until that ticket's slot is
 * submitted to again.  At most two waves may be submitted and not collected;
 * the GPU runs them in submission order, while the caller prepares the next or
 * consumes the last.  A cluster must not be in two uncollected waves.  The
 * first submit allocates a second set of wave buffers (abyss_ens_pipeline may
 * do it earlier).  While a wave is uncollected, set_wave, launch and fetch
 * refuse to touch its slot. */
int abyss_ens_pipeline(abyss_ens *e);
int abyss_ens_submit(abyss_ens *e, int nk, const int *clusters, const double *new_time, const double *time_scale,
                     const int *m_per, const int *targets_local, double eps2, int mode, int *ticket);
/* 1 when the wave of `ticket` and its result copies have finished, 0 if not yet. */
int abyss_ens_ready(abyss_ens *e, int ticket);
int abyss_ens_collect(abyss_ens *e, int ticket, const double **acc_reg, const double **jerk_reg,
                      const double **acc_irr, const double **jerk_irr, const int **nnb, const int **list,
                      int *rows, float *gpu_ms);
/* GPU milliseconds of the last launch (CUDA events around the wave). */
int abyss_ens_last_ms(abyss_ens *e, float *ms);
/* Rows, work items and kernel launches of the last wave. */
int abyss_ens_last_stats(const abyss_ens *e, int *rows, int *items, int *launches);

#ifdef __cplusplus
}
#endif
#endif
