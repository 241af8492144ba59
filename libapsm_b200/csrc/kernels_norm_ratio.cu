// Ratio of the linear to the Gaussian share of the model's norm, the
// reference's ApsmNomaDetector::computeNormRatio (cpp/lib/apsm/
// apsm_noma_detector.cu:220-311, public, no caller in the reference):
//   gaussian = wG sum_i sum_j a_i a_j k(d_i, d_j),  linear = wL sum_d w_d^2,
//   ratio = linear / gaussian,
// with k the Gaussian kernel of the detector (exp of the scaled squared
// distance, no weight).  Summed in the reference's order: row i by 32 lanes,
// lane t over j = t, t+32, ... (the product k a_i fused with a_j into the lane
// sum), lanes added in order, then rows in order; the linear sum in order.
// Dictionary rows are the detector's, oldest first (the reference's logical
// order).
#include "apsm_kernels.cuh"

namespace apsm {

namespace {

constexpr int kNrLanes = 32;

__global__ void __launch_bounds__(kNrLanes) norm_ratio_rows_kernel(const float* __restrict__ X, int Dp, int D, int M,
                                                                  const float* __restrict__ a, float ew,
                                                                  float* __restrict__ row_sums)
{
    const int i = blockIdx.x, t = threadIdx.x;
    __shared__ float part[kNrLanes];
    const float* xi = X + size_t(i) * Dp;
    const float ai = a[i];
    float acc = 0.f;
    for (int j = t; j < M; j += kNrLanes) {
        const float* xj = X + size_t(j) * Dp;
        float dist = 0.f;
        for (int d = 0; d < D; ++d) {
            const float diff = xi[d] - xj[d];
            dist = fmaf(diff, diff, dist);
        }
        acc = fmaf(expf(ew * dist) * ai, a[j], acc);
    }
    part[t] = acc;
    __syncthreads();
    if (t == 0) {
        float r = 0.f;
        for (int l = 0; l < kNrLanes && l < M; ++l) r += part[l];
        row_sums[i] = r;
    }
}

__global__ void norm_ratio_final_kernel(const float* __restrict__ row_sums, int M, const float* __restrict__ w, int D,
                                        float wL, float wG, float* __restrict__ out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float g = 0.f;
    for (int i = 0; i < M; ++i) g += row_sums[i];
    g *= wG;
    float l = 0.f;
    for (int d = 0; d < D; ++d) l = fmaf(w[d], w[d], l);
    l *= wL;
    out[0] = l / g;
}

} // namespace

cudaError_t launch_norm_ratio(const float* X, int Dp, int D, int M, const float* a, const float* w, float ew, float wL,
                              float wG, float* row_sums, float* out, cudaStream_t s)
{
    if (M > 0) {
        norm_ratio_rows_kernel<<<M, kNrLanes, 0, s>>>(X, Dp, D, M, a, ew, row_sums);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    norm_ratio_final_kernel<<<1, 1, 0, s>>>(row_sums, M, w, D, wL, wG, out);
    return cudaGetLastError();
}

} // namespace apsm
