// Tensor-core Gram detection (placeholder until the tcgen05 kernel lands).
#include "apsm_gram.cuh"

namespace apsm {
struct GramWorkspace {};
void gram_workspace_free(GramWorkspace* g) { delete g; }
} // namespace apsm

apsm_status detect_gram(apsm_detector* h, uint32_t, float*, cudaStream_t)
{
    h->last_error = "Gram detection is not available in this build";
    return APSM_ERR_UNSUPPORTED;
}
