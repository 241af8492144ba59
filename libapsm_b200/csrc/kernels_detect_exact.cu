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
// B200 layout, up to 16 features: the data rows and every feature of the
// warp's samples live in registers, dictionary tiles are staged feature-major
// in shared memory so a warp's 32 rows are read without bank conflicts.
// 32 to 128 features (detect_exact_wide_kernel): the block's samples sit in
// shared memory and are read as broadcast float4s, dictionary tiles arrive
// row-major by asynchronous copies (double-buffered) and each lane works on
// two rows for four samples at once, so eight independent distance chains
// hide the arithmetic latency and one dictionary load serves four samples.
// Either way the Gaussian value of each (sample, row) pair is computed once
// for all users of the cell (up to 16 per pass).
#include "apsm_kernels.cuh"

namespace apsm {

namespace {

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst))),
                 "l"(gmem_src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

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

// ----------------------------------------------------------- 32 to 128 features --
constexpr int kWideRows = 64;  // dictionary rows per tile: two per lane
constexpr int kWideSpw = 4;    // samples per warp
constexpr int kWideUsers = 16; // users per pass
constexpr int kWideSamples = kWarps * kWideSpw;

template <int DP> constexpr int wide_pitch() { return DP + 4; } // row pitch of a tile: float4 reads conflict-free

template <int DP> constexpr size_t wide_smem_bytes()
{
    return sizeof(float) * (size_t(2) * kWideRows * wide_pitch<DP>() + size_t(kWideSamples) * DP +
                            size_t(2) * kWideUsers * kWideRows);
}

template <int DP>
__global__ void __launch_bounds__(kWarps * 32, 2) detect_exact_wide_kernel(DetectArgs args)
{
    constexpr int P = wide_pitch<DP>();
    extern __shared__ __align__(16) float wsm[];
    float* tiles = wsm;                                  // [2][kWideRows][P]
    float* xs = tiles + 2 * kWideRows * P;               // [kWideSamples][DP]
    float* aws = xs + kWideSamples * DP;                 // [2][kWideUsers][kWideRows]

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int sb = blockIdx.x * kWideSamples;
    const int D = args.D, Dp = args.Dp, M = args.M;
    const int q4 = Dp >> 2;
    const ModelParams mp = args.mp;

    // the block's samples; features past Dp and samples past the end are zero
    for (int idx = tid; idx < kWideSamples * (DP / 4); idx += kWarps * 32) {
        const int r = idx / (DP / 4), c4 = idx - r * (DP / 4);
        float* dst = xs + r * DP + 4 * c4;
        if (sb + r < args.n_samples && c4 < q4) cp_async16(dst, args.Xs + size_t(sb + r) * Dp + 4 * c4);
        else *reinterpret_cast<float4*>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    // tile features past Dp stay zero (the copies never write them)
    for (int idx = tid; idx < 2 * kWideRows * (DP / 4 - q4); idx += kWarps * 32) {
        const int r = idx / (DP / 4 - q4), c4 = q4 + idx % (DP / 4 - q4);
        *reinterpret_cast<float4*>(tiles + r * P + 4 * c4) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    cp_async_commit();

    const int n_tiles = (M + kWideRows - 1) / kWideRows;
    const float* xw = xs + warp * kWideSpw * DP;
    for (int uc = 0; uc < args.users; uc += kWideUsers) {
        const int nu = min(kWideUsers, args.users - uc);
        // stage tile t: rows by asynchronous copies, coeff * gaussianKernelWeight (apsm_detect.cu:802) by plain stores
        auto stage = [&](int t) {
            const int b0 = t * kWideRows;
            float* tb = tiles + (t & 1) * kWideRows * P;
            for (int idx = tid; idx < kWideRows * q4; idx += kWarps * 32) {
                const int r = idx / q4, c4 = idx - r * q4;
                if (b0 + r < M) cp_async16(tb + r * P + 4 * c4, args.dict + size_t(b0 + r) * Dp + 4 * c4);
            }
            float* ab = aws + (t & 1) * kWideUsers * kWideRows;
            for (int idx = tid; idx < kWideUsers * kWideRows; idx += kWarps * 32) {
                const int u = idx / kWideRows, r = idx % kWideRows;
                const int b = b0 + r;
                ab[idx] = (u < nu && b < M) ? __fmul_rn(__ldg(args.a + size_t(uc + u) * args.a_stride + b), mp.wG) : 0.f;
            }
            cp_async_commit();
        };
        if (n_tiles > 0) stage(0);
        cp_async_wait<0>();
        __syncthreads(); // samples (and tile 0) in shared memory

        // linear part first (kernel_apsm_detection_linear_shmem)
        float p[kWideSpw][kWideUsers];
#pragma unroll
        for (int s = 0; s < kWideSpw; ++s) {
#pragma unroll
            for (int u = 0; u < kWideUsers; ++u) p[s][u] = 0.f;
            for (int idx = lane; idx < D; idx += 32) {
                const float ke = __fmul_rn(mp.wL, xw[s * DP + idx]);
#pragma unroll
                for (int u = 0; u < kWideUsers; ++u)
                    if (u < nu) p[s][u] = __fadd_rn(p[s][u], __fmul_rn(__ldg(args.w + size_t(uc + u) * D + idx), ke));
            }
        }

        for (int t = 0; t < n_tiles; ++t) {
            if (t + 1 < n_tiles) {
                stage(t + 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads(); // tile t complete for every thread
            const float* tb = tiles + (t & 1) * kWideRows * P;
            const float* ab = aws + (t & 1) * kWideUsers * kWideRows;
            // lane rows r0 = lane, r1 = lane + 32: the lane's rows b = lane + 32 j in ascending order
            float acc[2][kWideSpw];
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int s = 0; s < kWideSpw; ++s) acc[h][s] = 0.f;
            const float* d0 = tb + lane * P;
            const float* d1 = tb + (lane + 32) * P;
#pragma unroll 4
            for (int c = 0; c < DP; c += 4) {
                const float4 v0 = *reinterpret_cast<const float4*>(d0 + c);
                const float4 v1 = *reinterpret_cast<const float4*>(d1 + c);
#pragma unroll
                for (int s = 0; s < kWideSpw; ++s) {
                    const float4 xv = *reinterpret_cast<const float4*>(xw + s * DP + c);
                    float e;
                    e = v0.x - xv.x; acc[0][s] = fmaf(e, e, acc[0][s]);
                    e = v1.x - xv.x; acc[1][s] = fmaf(e, e, acc[1][s]);
                    e = v0.y - xv.y; acc[0][s] = fmaf(e, e, acc[0][s]);
                    e = v1.y - xv.y; acc[1][s] = fmaf(e, e, acc[1][s]);
                    e = v0.z - xv.z; acc[0][s] = fmaf(e, e, acc[0][s]);
                    e = v1.z - xv.z; acc[1][s] = fmaf(e, e, acc[1][s]);
                    e = v0.w - xv.w; acc[0][s] = fmaf(e, e, acc[0][s]);
                    e = v1.w - xv.w; acc[1][s] = fmaf(e, e, acc[1][s]);
                }
            }
            const int bt = t * kWideRows;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = lane + 32 * h;
                if (bt + r < M) {
#pragma unroll
                    for (int s = 0; s < kWideSpw; ++s) {
                        const float kv = expf(__fmul_rn(mp.ew, acc[h][s]));
#pragma unroll
                        for (int u = 0; u < kWideUsers; ++u)
                            if (u < nu) p[s][u] = __fadd_rn(p[s][u], __fmul_rn(ab[u * kWideRows + r], kv));
                    }
                }
            }
            __syncthreads(); // buffer t & 1 is restaged by iteration t + 1
        }
        // warp shuffle-down tree (apsm_detect.cu:830-833)
#pragma unroll
        for (int s = 0; s < kWideSpw; ++s) {
            const int si = sb + warp * kWideSpw + s;
#pragma unroll
            for (int u = 0; u < kWideUsers; ++u) {
                float acc = p[s][u];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) acc = __fadd_rn(acc, __shfl_down_sync(0xffffffffu, acc, off));
                if (lane == 0 && u < nu && si < args.n_samples) args.out[size_t(uc + u) * args.out_stride + si] = acc;
            }
        }
    }
}

template <int DP>
void launch_wide(const DetectArgs& args, cudaStream_t stream)
{
    // above the 48 KB default: opt in (per device, so on every launch)
    if (cudaFuncSetAttribute(detect_exact_wide_kernel<DP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(wide_smem_bytes<DP>())) != cudaSuccess)
        return; // the error stays for the caller's cudaGetLastError
    const int grid = (args.n_samples + kWideSamples - 1) / kWideSamples;
    detect_exact_wide_kernel<DP><<<grid, kWarps * 32, wide_smem_bytes<DP>(), stream>>>(args);
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
    else if (args.D <= 32) launch_wide<32>(args, stream);
    else if (args.D <= 64) launch_wide<64>(args, stream);
    else launch_wide<128>(args, stream);
}

} // namespace apsm
