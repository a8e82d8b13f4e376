/* abyss_io.h -- state I/O of the host integrator (libabyss_reg.so): the
 * reference's text formats, and a restartable binary checkpoint.
 *
 * Text formats (src_mpi/ReadWrite.cpp:20-97 reads, :140-245 writes; unit
 * conversions of src_mpi/particle.h:139-147,204-214 and src_mpi/def.h:51-60):
 *   input   one particle per line: x y z [kpc], vx vy vz [km/s], mass [1e9 Msun];
 *           every line is a particle, missing columns read as 0;
 *   output  "<t> Myr," / "<output time>, <output step>, <code time>" / a column
 *           header / one row per particle: PID, mass [Msun], x y z [pc],
 *           vx vy vz [km/s], 18-wide columns, fixed with 8 decimals, positions
 *           and velocities predicted to the snapshot time.
 * Code units are the reference's: G = 1 with 4 pc, 4e-10 pc/yr and
 * 1.424198e-4 Msun.
 */
#ifndef ABYSS_IO_H
#define ABYSS_IO_H
#ifdef __cplusplus
extern "C" {
#endif

struct abyss_ac;
struct abyss_ctx;

/* Read a reference input file into code units.  Call with x = v = mass = NULL
 * to get the particle count in *n, then with arrays of *n ([n][3], [n][3], [n]). */
int abyss_read_reference_ic(const char *path, int *n, double *x, double *v, double *mass);

/* Write the integrator's state as a reference snapshot (writeParticle of
 * ReadWrite.cpp); output_time and output_time_step fill the second header line. */
int abyss_ac_write_snapshot(const struct abyss_ac *ac, const char *path, double output_time,
                            double output_time_step);

/* Checkpoint: every field of the integration (particles, derivatives, neighbour
 * lists, block times and steps, parameters, statistics) in a native-endian
 * binary file.  Only between regular blocks (ABYSS_ERR_STATE while one is open).
 * abyss_ac_load rebuilds the integration on ctx without recomputing anything,
 * so that continuing it gives the same results, bit for bit, as never having
 * stopped; threads replaces the saved host thread count.  A file that is not a
 * complete checkpoint of this version is refused with ABYSS_ERR_STATE, before
 * any allocation where its particle count exceeds what its size can hold; a
 * failed host allocation returns ABYSS_ERR_OOM.  ctx may
 * be NULL: the integration then serves host-side calls only (state queries, the
 * irregular steps of abyss_ac_begin_block, abyss_ac_save); calls that need the
 * GPU return ABYSS_ERR_ARG. */
int abyss_ac_save(const struct abyss_ac *ac, const char *path);
int abyss_ac_load(struct abyss_ctx *ctx, const char *path, int threads, struct abyss_ac **out);

#ifdef __cplusplus
}
#endif
#endif
