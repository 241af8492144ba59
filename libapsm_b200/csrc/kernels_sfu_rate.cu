// Measured exponential throughput of the SFU: the denominator of the
// detection stage's roofline.  Every exponential of the detection kernels is
// one ex2.approx.ftz.f32 (base 2, arguments pre-scaled by log2 e); this
// kernel issues nothing else of weight: eight independent chains per thread of
// v <- 2^v - 1 (v stays in [-1, 0]: no denormals, no infinities), eight
// 256-thread CTAs per SM, timed with CUDA events after a warm-up launch.
#include "apsm_b200.h"
#include "apsm_tc.cuh"

#include <cuda_runtime.h>

namespace apsm {

namespace {

constexpr int kChains = 8;
constexpr int kThreadsSfu = 256;

__global__ void __launch_bounds__(kThreadsSfu) sfu_rate_kernel(float* out, int iters)
{
    float v[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = -1e-3f * float((threadIdx.x + 37 * c) & 1023);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) v[c] = tc::ex2(v[c]) - 1.0f;
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += v[c];
    if (s > 1.0f) out[blockIdx.x] = s; // never true (v <= 0): keeps the chains live without a store per thread
}

} // namespace

} // namespace apsm

extern "C" apsm_status apsm_measure_ex2_rate(double* per_second, float* ms)
{
    using namespace apsm;
    if (!per_second) return APSM_ERR_INVALID_ARGUMENT;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return APSM_ERR_NO_DEVICE;
    }
    float* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t s = nullptr;
    apsm_status st = APSM_OK;
    const int grid = 8 * sms, iters = 4096;
    float t = 0.f;
    if (cudaMalloc(&out, sizeof(float) * grid) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess || cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        st = APSM_ERR_CUDA;
    } else {
        sfu_rate_kernel<<<grid, kThreadsSfu, 0, s>>>(out, iters); // warm-up (clocks up, code loaded)
        cudaEventRecord(e0, s);
        sfu_rate_kernel<<<grid, kThreadsSfu, 0, s>>>(out, iters);
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess || t <= 0.f)
            st = APSM_ERR_CUDA;
    }
    if (st == APSM_OK) {
        *per_second = double(grid) * kThreadsSfu * double(iters) * kChains / (double(t) * 1e-3);
        if (ms) *ms = t;
    }
    cudaGetLastError();
    if (s) cudaStreamDestroy(s);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (out) cudaFree(out);
    return st;
}
