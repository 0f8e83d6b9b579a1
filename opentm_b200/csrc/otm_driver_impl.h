// otm_driver_impl.h -- device helpers shared by the initialisers and the design loop (internal).
#pragma once

#include <cuda_runtime.h>

#include "opentm_b200.h"

namespace otm {

// Orbit means of a pitched field under an OTM_SYM_* group (launches only).
otm_status symmetrize_field(const int reso[3], float* f, int pitchT, int sym, int average, cudaStream_t s);
// Means of two pitched fields (FP64, fixed reduction order); waits for the stream.
otm_status field_means(const int reso[3], const float* a, const float* b, int pitchT, cudaStream_t s, double out[2]);

}  // namespace otm
