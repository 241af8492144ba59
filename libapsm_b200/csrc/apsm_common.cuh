// Shared definitions of the B200 APSM kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace apsm {

constexpr int kLanes = 32;        // reference lane partition (APSM_BLOCK_BATCH_SIZE, cuda_indexing.cuh:74)
constexpr int kMaxFeatures = 128; // D = 2N real features, N <= 64 antennas
constexpr int kWGroups = 8;       // linear-weight update: window terms summed in 8 interleaved groups

// Scalar model parameters as the kernels see them.  Values are the reference's
// float parameters (apsm_parameters.cuh:68-86) after the constructor's
// variance scaling (apsm_noma_detector.cu:79-80).
struct ModelParams {
    float wL;  // linearKernelWeight = 1 - gaussianKernelWeight
    float wG;  // gaussianKernelWeight
    float ew;  // exp weight -0.5f / gaussianKernelVariance (apsm_detect.cu:135)
    float eB;  // hyperslab half width
};

// One step of the training schedule (host step loop apsm_train.cu:107-160):
// visible dictionary rows are [max(0, hi - cap), hi) in universe order, the
// projection window is [hi - wk, hi) and its first n_active rows are updated.
struct TrainStep {
    int hi;
    int wk;
    int n_active;
    int reveal_lo; // rows [reveal_lo, hi) become visible at this step (a = 0)
};

__host__ __device__ inline uint32_t round_up(uint32_t x, uint32_t m) { return (x + m - 1) / m * m; }

// Limit (ns) of the bounded barrier waits of the tensor-core kernels, read by
// their launchers (apsm_set_wait_limit_ns; 2 s unless changed).
unsigned long long wait_limit_ns();

// Row pitch (floats) of dictionary / sample rows in HBM: D padded to 4 so
// that every row starts 16-byte aligned.
__host__ __device__ inline uint32_t row_pitch(uint32_t D) { return round_up(D, 4); }

} // namespace apsm
