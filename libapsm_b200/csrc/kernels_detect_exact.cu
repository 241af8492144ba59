// Exact FP32 APSM detection (the "plain" form): the model
//   f(x_s) = wL <w, x_s> + sum_b (a_b wG) exp(ew ||d_b - x_s||^2)
// evaluated in the reference BALANCED kernel's order
// (cpp/lib/apsm/apsm_detect.cu:526-538 linear part, :690-808 Gaussian part,
// :810-876 reduction): lane l of the warp that owns sample s accumulates
// first the linear terms idx = l, l+32, ... and then the Gaussian terms of
// dictionary rows b = l, l+32, ... in ascending order; squared distances are
// sequential fma chains over the features; the 32 partials are combined with
// the shuffle-down tree.  Given the same coefficients the soft outputs are
// bit-identical to the reference's.
//
// B200 layout: the data rows and every feature of the warp's samples live in
// registers, dictionary tiles are staged feature-major in shared memory so a
// warp's 32 rows are read without bank conflicts, and the Gaussian value of
// each (sample, row) pair is computed once for all users of the cell.
#include "apsm_kernels.cuh"

namespace apsm {

namespace {

constexpr int kUserChunk = 8;     // users accumulated per pass
constexpr int kWarps = 8;

// dictionary rows per shared-memory tile (static shared memory stays below 48 KB)
template <int DP> constexpr int tile_rows() { return DP >= 128 ? 64 : 128; }

template <int DP, int SPW>
__global__ void __launch_bounds__(kWarps * 32) detect_exact_kernel(DetectArgs args)
{
    constexpr int kTileRows = tile_rows<DP>();
    __shared__ float dT[DP][kTileRows + 1];
    __shared__ float aw[kUserChunk][kTileRows];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int s0 = (blockIdx.x * kWarps + warp) * SPW;
    const int D = args.D, Dp = args.Dp, M = args.M;
    const ModelParams mp = args.mp;

    float x[SPW][DP];
#pragma unroll
    for (int s = 0; s < SPW; ++s) {
        const int si = s0 + s;
#pragma unroll
        for (int d = 0; d < DP; ++d)
            x[s][d] = (si < args.n_samples && d < D) ? __ldg(args.Xs + size_t(si) * Dp + d) : 0.f;
    }

    for (int uc = 0; uc < args.users; uc += kUserChunk) {
        const int nu = min(kUserChunk, args.users - uc);
        float p[SPW][kUserChunk];
        // linear part first (kernel_apsm_detection_linear_shmem)
#pragma unroll
        for (int s = 0; s < SPW; ++s) {
#pragma unroll
            for (int u = 0; u < kUserChunk; ++u) p[s][u] = 0.f;
            const int si = s0 + s;
            if (si < args.n_samples) {
                for (int idx = lane; idx < D; idx += 32) {
                    const float ke = __fmul_rn(mp.wL, __ldg(args.Xs + size_t(si) * Dp + idx));
#pragma unroll
                    for (int u = 0; u < kUserChunk; ++u)
                        if (u < nu) p[s][u] = __fadd_rn(p[s][u], __fmul_rn(__ldg(args.w + size_t(uc + u) * D + idx), ke));
                }
            }
        }
        // Gaussian part over dictionary tiles
        for (int b0 = 0; b0 < M; b0 += kTileRows) {
            __syncthreads();
            for (int idx = threadIdx.x; idx < kTileRows * DP; idx += kWarps * 32) {
                const int r = idx / DP, d = idx % DP;
                const int b = b0 + r;
                dT[d][r] = (b < M && d < D) ? __ldg(args.dict + size_t(b) * Dp + d) : 0.f;
            }
            for (int idx = threadIdx.x; idx < kUserChunk * kTileRows; idx += kWarps * 32) {
                const int u = idx / kTileRows, r = idx % kTileRows;
                const int b = b0 + r;
                // coeff(b) * gaussianKernelWeight (apsm_detect.cu:802)
                aw[u][r] = (u < nu && b < M) ? __fmul_rn(__ldg(args.a + size_t(uc + u) * args.a_stride + b), mp.wG) : 0.f;
            }
            __syncthreads();
#pragma unroll 1
            for (int k = 0; k < kTileRows / 32; ++k) {
                const int r = k * 32 + lane;
                if (b0 + r >= M) break;
#pragma unroll
                for (int s = 0; s < SPW; ++s) {
                    float acc = 0.f;
#pragma unroll
                    for (int d = 0; d < DP; ++d) {
                        const float diff = dT[d][r] - x[s][d];
                        acc = fmaf(diff, diff, acc);
                    }
                    const float kv = expf(__fmul_rn(mp.ew, acc));
#pragma unroll
                    for (int u = 0; u < kUserChunk; ++u)
                        if (u < nu) p[s][u] = __fadd_rn(p[s][u], __fmul_rn(aw[u][r], kv));
                }
            }
        }
        // warp shuffle-down tree (apsm_detect.cu:830-833)
#pragma unroll
        for (int s = 0; s < SPW; ++s) {
#pragma unroll
            for (int u = 0; u < kUserChunk; ++u) {
                float acc = p[s][u];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) acc = __fadd_rn(acc, __shfl_down_sync(0xffffffffu, acc, off));
                const int si = s0 + s;
                if (lane == 0 && u < nu && si < args.n_samples) args.out[size_t(uc + u) * args.out_stride + si] = acc;
            }
        }
    }
}

template <int DP, int SPW>
void launch_dp(const DetectArgs& args, cudaStream_t stream)
{
    const int per_block = kWarps * SPW;
    const int grid = (args.n_samples + per_block - 1) / per_block;
    detect_exact_kernel<DP, SPW><<<grid, kWarps * 32, 0, stream>>>(args);
}

} // namespace

void launch_detect_exact(const DetectArgs& args, cudaStream_t stream)
{
    if (args.n_samples <= 0) return;
    if (args.D <= 8) launch_dp<8, 4>(args, stream);
    else if (args.D <= 16) launch_dp<16, 4>(args, stream);
    else if (args.D <= 32) launch_dp<32, 2>(args, stream);
    else if (args.D <= 64) launch_dp<64, 1>(args, stream);
    else launch_dp<128, 1>(args, stream);
}

} // namespace apsm
