// Tensor-core (tcgen05) Gram detection: entry points used by the detector.
#pragma once

#include "apsm_host.hpp"

namespace apsm {
void gram_workspace_free(GramWorkspace* g);
} // namespace apsm

// Detection of the packed data rows h->xs (2S rows) with the Gram form
// selected by h->cfg.detect_mode; soft outputs to d_out (users x 2S floats).
apsm_status detect_gram(apsm_detector* h, uint32_t S, float* d_out, cudaStream_t s);
// Expiry of a bounded wait in the last Gram detection of h (read after its
// stream synchronised): APSM_ERR_CUDA once, then cleared.
apsm_status detect_gram_check(apsm_detector* h);
