// Host-side launch wrappers of the kernels in kernels.cu.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "abyss_internal.cuh"

namespace abyss {

void launch_predict(cudaStream_t s, int n, const double *x, const double *v, const double *a0,
                    const double *a1, const double *t0, const double *mass, double new_time,
                    double time_scale, double *px, double *py, double *pz, double *pvx,
                    double *pvy, double *pvz, float4 *vm, int sm_count);
void launch_pack_vm(cudaStream_t s, int n, const double *pvx, const double *pvy, const double *pvz,
                    const double *mass, float4 *vm, int sm_count);
void launch_unpack_predicted(cudaStream_t s, int n, const double *pos, const double *vel,
                             const double *mass, double *px, double *py, double *pz, double *pvx,
                             double *pvy, double *pvz, float4 *vm, int sm_count);
void launch_iota(cudaStream_t s, int m, int *out, int sm_count);
size_t sort_temp_bytes(int m_cap);
// Spatial order of the targets (Hilbert key of their positions, stable radix
// sort) into order_t/order_o; with `anchor`, also the bounding-box centre of
// every i-block of per_block consecutive slots ([nblk][3] doubles).
void launch_spatial_order(cudaStream_t s, int m, const int *targets, const JSet &js, int *bbox,
                          uint32_t *keys, uint32_t *keys_alt, int *rows, int *rows_alt, void *cub_tmp,
                          size_t cub_bytes, int *order_t, int *order_o, int per_block, double *anchor,
                          int sm_count);
int tile_occupancy(int nt, int ipt, bool anchor, bool pack, int unr, int minb);
int launch_tile(cudaStream_t s, int nt, int ipt, bool anchor, bool pack, int unr, int minb, int grid,
                const JSet &js, const Work &w, int n_iblocks);
// Tile kernel whose 4 warps share a block's 32 x ipt targets (ipt 1 or 2) and
// split each j-tile between them (abyss_tuning.kernel = 4); unr j per step (1, 2).
int tile_split_occupancy(int ipt, int unr, bool packed);
int launch_tile_split(cudaStream_t s, int ipt, int unr, bool packed, int grid, const JSet &js, const Work &w,
                      int n_iblocks);
int tile_variant_count();
int tile_variant_shape(int i, int *shape6);
// j-major force kernel: w.n_chunks blocks of jmajor_warps() warps, each warp a
// sub-chunk of Lw particles (a multiple of 64).
int jmajor_warps();
int jmajor_occupancy(int mi);  // resident blocks per SM
// With `fuse` (few rows), the last block to finish also finalizes the rows into
// *fuse, in place of launch_finalize; w.item_counter must be zero.
int launch_jmajor(cudaStream_t s, int mi, const JSet &js, const Work &w, int Lw, const Outputs *fuse = nullptr);
void launch_finalize(cudaStream_t s, const JSet &js, const Work &w, const Outputs &o, int sm_count);
void launch_predict_multi(cudaStream_t s, int n, const int *cid, const int *active,
                          const double *new_time, const double *time_scale, const double *x,
                          const double *v, const double *a0, const double *a1, const double *t0,
                          const double *mass, double *px, double *py, double *pz, double *pvx,
                          double *pvy, double *pvz, float4 *vm, int sm_count);
void launch_finalize_grid(cudaStream_t s, const JSet &js, const Work &w, const Outputs &o, int blocks);
void launch_energy(cudaStream_t s, int n, const double *x, const double *v, const double *mass,
                   double eps2, double *e_row);
// init_derivs.cu: out [n][12] = (reg2, reg3, irr2, irr3) x 3 dimensions
void launch_init_derivs23(cudaStream_t s, int n, const double *x, const double *v, const double *a0,
                          const double *a1, const double *mass, const double *r2nb, double eps2,
                          double *out);

}  // namespace abyss

struct abyss_ctx;
namespace abyss {
cudaStream_t ctx_stream(abyss_ctx *c);
int ctx_device(abyss_ctx *c);
int ctx_sm_count(abyss_ctx *c);
}  // namespace abyss
