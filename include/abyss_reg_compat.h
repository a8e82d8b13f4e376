/* abyss_reg_compat.h -- drop-in for the reference's GPU regular-force ABI.
 *
 * Same names, arguments and meaning as src_mpi/cuda/cuda_functions.h:3-10
 * (CUDA_REAL = float, src_mpi/def.h:69-72) and, with the _f64 suffix, as
 * src/cuda/cuda_functions.h:3-10 (CUDA_REAL = double, src/defs.h:97-102).
 * Implemented in libabyss_reg.so on top of abyss_reg.h.
 *
 * Behaviour kept from the reference (src_mpi/cuda/cuda_my_acceleration.cu):
 *   - SendToDevice takes the already predicted j-set (x, v [NNB][3], masses,
 *     squared neighbour radii r2); mdot is ignored (:603-778).
 *   - CalculateAccelerationOnDevice takes NumTarget indices into that j-set
 *     and returns the regular acc/adot (neighbours excluded), neighbour
 *     counts and lists in ascending index, rows NeighborList[i*stride ..],
 *     stride = NumNeighborMax of the caller's build (1000 for src_mpi, 200
 *     for src; set with abyss_compat_set_list_stride) (:95-344, :1087-1106).
 *   - No softening (the reference's GPU path has none).
 * Differences (documented, deliberate):
 *   - Neighbour test is the reference CPU rule r2 < R2 in FP64
 *     (ComputeAcceleration.cpp:285), not the GPU kernel's FP32 !(r2 > R2)
 *     (cuda_kernels.cu:338,361).
 *   - A list longer than the stride never traps the GPU (the reference
 *     asserts in device code, cuda_kernels.cu:363,432): NumNeighbor holds the
 *     exact count, the row is truncated, a message goes to stderr and
 *     abyss_compat_status() returns ABYSS_WARN_OVERFLOW.
 *   - One GPU (the reference splits j over up to four, :119-281).
 */
#ifndef ABYSS_REG_COMPAT_H
#define ABYSS_REG_COMPAT_H
#ifdef __cplusplus
extern "C" {
#endif

/* cuda_functions.h:4 -- select and initialise the device (irank % devices). */
void InitializeDevice(int *irank);
/* cuda_functions.h:5 -- InitializeDevice + mark open (warns if already open). */
void OpenDevice(const int *irank);
/* cuda_functions.h:6 -- mark closed and free the library's device memory. */
void CloseDevice(void);
/* cuda_functions.h:7 -- print call/pair/time counters when ABYSS_PROFILE is set. */
void ProfileDevice(int *irank);
/* cuda_functions.h:8 -- upload the predicted j-set (FP32 spelling). */
void SendToDevice(int *NNB, float m[], float x[][3], float v[][3], float r2[], float mdot[]);
/* cuda_functions.h:9 -- regular acc/adot + neighbour lists (FP32 spelling). */
void CalculateAccelerationOnDevice(int *NumTarget, int *h_target_list, float acc[][3],
                                   float adot[][3], int NumNeighbor[], int *NeighborList);
/* src/cuda/cuda_functions.h:8 with CUDA_REAL = double. */
void SendToDevice_f64(int *NNB, double m[], double x[][3], double v[][3], double r2[],
                      double mdot[]);
/* src/cuda/cuda_functions.h:9 with CUDA_REAL = double. */
void CalculateAccelerationOnDevice_f64(int *NumTarget, int *h_target_list, double acc[][3],
                                       double adot[][3], int NumNeighbor[], int *NeighborList);

/* Row stride of NeighborList (the caller's NumNeighborMax); default 1000. */
int abyss_compat_set_list_stride(int stride);
/* Status of the last compat call: ABYSS_OK, ABYSS_WARN_OVERFLOW or ABYSS_ERR_*. */
int abyss_compat_status(void);

#ifdef __cplusplus
}
#endif
#endif
