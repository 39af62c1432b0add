// Launch interface of the wavefront path tracer (wavefront.cu).
#pragma once
#include "kernels.h"

// Device scratch bytes for `slots` concurrent paths.
size_t pt_wavefront_bytes(uint32_t slots);

// Renders the frame described by p with up to `slots` paths in flight, using
// `scratch` (pt_wavefront_bytes(slots) bytes of device memory). Blocks: the
// host reads the ray-queue length back every few waves to know when the
// frame is done. host_counts: 4 bytes of pinned host memory.
cudaError_t pt_launch_wavefront(const PtSceneDev& scene, const PtRenderParams& p, void* scratch, uint32_t slots,
                                int sms, cudaStream_t stream, uint32_t* host_counts);
