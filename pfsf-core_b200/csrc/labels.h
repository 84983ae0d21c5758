// Island labelling (labels.cu).
#pragma once
#include <cuda_runtime.h>

#include "pfsf/pfsf.h"

namespace pfsf_b200 {
namespace labels {
// 26-connected components of the non-air voxels of an lx*ly*lz box on
// stream s; see pfsf_label_components in pfsf_b200.h for the outputs.
pfsf_result label_components(cudaStream_t s, int num_sms, const uint8_t* host_type, int32_t lx, int32_t ly, int32_t lz,
                             uint32_t* host_labels, pfsf_label_component* host_comps, int32_t capacity,
                             int32_t* out_count, int32_t* out_overflow);
}  // namespace labels
}  // namespace pfsf_b200
