// Internal interface between a regular-force context (context.cu) and the host
// integrator's whole regular blocks on the device (host/ac_integrator.cpp):
// the j-set state, the targets and the results stay in device memory.
#pragma once
#include <cuda_runtime.h>

#include "irregular.h"

struct abyss_ctx;

namespace abyss {
cudaStream_t ctx_stream(abyss_ctx *c);
int ctx_device(abyss_ctx *c);
int ctx_wait_spin(abyss_ctx *c);  // the wait policy of abyss_set_wait (< 0: stream synchronisation)
int ctx_state_buffers(abyss_ctx *c, int n, abyss_irr::JsetDst *d);
int ctx_targets_from_device(abyss_ctx *c, int m, const int *d_targets);
int ctx_launch_status(abyss_ctx *c, int *status, int *ovf);
int ctx_results(abyss_ctx *c, abyss_irr::RegResults *r);
int ctx_read_targets(abyss_ctx *c, int *targets, double *r2nb);
}  // namespace abyss
