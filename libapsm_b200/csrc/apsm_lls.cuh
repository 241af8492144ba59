// Linear least-squares detector (kernels_lls.cu).
#pragma once

#include "apsm_host.hpp"

namespace apsm {
struct LlsWorkspace;
void lls_workspace_free(LlsWorkspace* l);
apsm_status lls_solve(apsm_detector* h, const float* rows, int n, const float* y, size_t y_stride, int row0,
                      float divide_by, cudaStream_t s);
apsm_status lls_detect(apsm_detector* h, int ns, float* d_out, cudaStream_t s);
const float* lls_weights(apsm_detector* h);
} // namespace apsm
