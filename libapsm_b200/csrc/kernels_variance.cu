// Gaussian-variance heuristic on the GPU: the reference's
// computeGaussianVarianceHeuristic (cpp/lib/apsm/apsm_noma_detector.cu:193-218,
// host code there, used when gaussianKernelVariance is 0):
//   for every pair of pilots i < j:  d_ij = sqrt(sum_k |y_k,i - y_k,j|)
//   (float sum over antennas in order, |.| the complex modulus), then
//   variance = (d_(0.7 M) * P^(-1/5))^2 with d_(r) the r-th smallest of the
//   M = P (P-1) / 2 values.
// The modulus is formed as the C library forms it for float complex numbers
// (squares and sum in double, square root in double, rounded to float), so
// the distances are those of the reference's host code bit for bit; the
// order statistic is found exactly by a radix select over the float bit
// patterns (non-negative floats order like their bits): four passes of a
// 256-bucket histogram, each narrowing the prefix of the wanted value.
#include "apsm_b200.h"
#include "apsm_kernels.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

namespace apsm {

namespace {

__global__ void __launch_bounds__(256) pair_distance_kernel(const float2* __restrict__ rx, int N, int P,
                                                            float* __restrict__ nd)
{
    // pair index -> (i, j), i < j: row i holds pairs [i P - i (i+1) / 2, ...)
    const long long M = (long long)P * (P - 1) / 2;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < M;
         q += (long long)gridDim.x * blockDim.x) {
        // smallest i with start(i + 1) > q, start(i) = i P - i (i + 1) / 2
        const double b = 2.0 * P - 1.0;
        long long i = (long long)((b - sqrt(b * b - 8.0 * double(q))) / 2.0);
        if (i < 0) i = 0;
        while (i > 0 && i * P - i * (i + 1) / 2 > q) --i;
        while ((i + 1) * P - (i + 1) * (i + 2) / 2 <= q) ++i;
        const long long j = q - (i * P - i * (i + 1) / 2) + i + 1;
        float dist = 0.f;
        for (int k = 0; k < N; ++k) {
            const float2 u = rx[size_t(k) * P + i], v = rx[size_t(k) * P + j];
            const double re = double(__fsub_rn(u.x, v.x)), im = double(__fsub_rn(u.y, v.y));
            const float m = __double2float_rn(__dsqrt_rn(__dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im))));
            dist = __fadd_rn(dist, m);
        }
        nd[q] = __fsqrt_rn(dist);
    }
}

// 256-bucket histogram of bits [shift, shift + 8) of the values whose bits above
// shift + 8 equal `prefix` (all values when shift == 24)
__global__ void __launch_bounds__(256) radix_hist_kernel(const float* __restrict__ nd, long long M, int shift,
                                                         unsigned prefix, unsigned long long* __restrict__ hist)
{
    __shared__ unsigned h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const unsigned hi_mask = shift >= 24 ? 0u : (0xffffffffu << (shift + 8));
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < M; q += (long long)gridDim.x * blockDim.x) {
        const unsigned u = __float_as_uint(nd[q]);
        if ((u & hi_mask) == (prefix & hi_mask)) atomicAdd(&h[(u >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    if (h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], (unsigned long long)h[threadIdx.x]);
}

} // namespace

apsm_status variance_heuristic_gpu(const float2* d_rx, uint32_t N, uint32_t P, float* d_nd,
                                   unsigned long long* d_hist, cudaStream_t s, float* variance, std::string* err)
{
    const long long M = (long long)P * (P - 1) / 2;
    if (M <= 0) {
        *variance = 0.f;
        return APSM_OK;
    }
    auto ck = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess) *err = std::string(what) + ": " + cudaGetErrorString(e);
        return e == cudaSuccess;
    };
    const int blocks = int(std::min<long long>((M + 255) / 256, 148LL * 16));
    pair_distance_kernel<<<blocks, 256, 0, s>>>(d_rx, int(N), int(P), d_nd);
    if (!ck(cudaGetLastError(), "pair_distance_kernel")) return APSM_ERR_CUDA;
    // index of the reference: normDistances[size * p], size * p in float
    const long long idx = (long long)(float(M) * 0.7f);
    long long rank = idx; // rank of the wanted value among those matching the prefix
    unsigned prefix = 0;
    unsigned long long h[256];
    for (int shift = 24; shift >= 0; shift -= 8) {
        if (!ck(cudaMemsetAsync(d_hist, 0, sizeof(h), s), "cudaMemsetAsync")) return APSM_ERR_CUDA;
        radix_hist_kernel<<<blocks, 256, 0, s>>>(d_nd, M, shift, prefix, d_hist);
        if (!ck(cudaGetLastError(), "radix_hist_kernel")) return APSM_ERR_CUDA;
        if (!ck(cudaMemcpyAsync(h, d_hist, sizeof(h), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync")) return APSM_ERR_CUDA;
        if (!ck(cudaStreamSynchronize(s), "cudaStreamSynchronize")) return APSM_ERR_CUDA;
        int b = 0;
        while (b < 255 && rank >= (long long)h[b]) rank -= (long long)h[b++];
        prefix |= unsigned(b) << shift;
    }
    float nd_idx;
    std::memcpy(&nd_idx, &prefix, sizeof(nd_idx));
    // variance = nd[idx] * pow(P, -1 / q) in double, stored as float, then squared in float
    float v = float(double(nd_idx) * std::pow(double(P), -1.0 / double(5.0f)));
    *variance = v * v;
    return APSM_OK;
}

} // namespace apsm
