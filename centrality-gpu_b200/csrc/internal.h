// Library-internal helpers shared between translation units (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include "bcgpu.h"

namespace bcg {

// Device, stream and the two timing events a context owns.
void ctx_device_stream(const bc_ctx *ctx, int *device, cudaStream_t *stream, cudaEvent_t *ev0, cudaEvent_t *ev1);
// Records msg as the context's last error (read back by bc_last_error).
void ctx_set_error(bc_ctx *ctx, const char *msg);
// The text and the BCGPU_* status of a device error code (common.cuh DevErr),
// shared by every entry point that reads a kernel's error flag.
const char *dev_err_text(int code);
int dev_err_status(int code);

// Profiling builds only (-DBCGPU_HOST_TIMERS): prints the wall time since
// the previous mark under `name` to stderr (one plan build at a time).
#ifdef BCGPU_HOST_TIMERS
void host_mark(const char *name);
#define HOST_MARK(n) ::bcg::host_mark(n)
#else
#define HOST_MARK(n) do {} while (0)
#endif
}  // namespace bcg
