// Kernel columns of the batched training sweep, all jobs in one launch.
//
// For every pair n that enters a window during the sweep, column n holds,
// against every pair b the sweep may combine with n (b in
// [max(0, n + 1 - capP), min(n + qP, nP))), the three distinct values of the
// combined kernel Kt = K + wL <x, x'> (Gaussian plus weighted linear kernel):
// (A + wL r, Bp + wL m, Bm - wL m) with r + i m = y_b^H y_n.  Same
// quantities as the reference's per-evaluation distance loop
// (cpp/lib/apsm/apsm_detect.cu:131-152) and linear kernel (:103-129), formed
// from y_b^H y_n and the row norms.
#include "apsm_batch.cuh"

namespace apsm {

namespace {

constexpr int kColGroup = kKcolGroup; // columns per block
constexpr int kColRows = kKcolRows;   // column entries per block pass (= threads)

__global__ void __launch_bounds__(kColRows)
    batch_kcol_kernel(const BatchTrainJob* __restrict__ jobs, BatchCommon cm, int smem_n)
{
    const BatchTrainJob& jb = jobs[blockIdx.y];
    const int nP = jb.nP, N = jb.N, Np = jb.Np, capP = jb.capP, qP = cm.qP;
    const int n0 = jb.n_first + blockIdx.x * kColGroup;
    if (n0 >= nP || N > smem_n) return; // shared memory is sized for smem_n antennas
    const int nc = min(kColGroup, nP - n0);
    const float ew = jb.ew, wG = cm.wG, wL = cm.wL;
    const int tid = threadIdx.x;

    extern __shared__ float2 smk[];
    constexpr int kPitch = kColRows + 1;
    float2* sY = smk;                         // [N][kPitch] feature-major universe pairs
    float2* sC = sY + size_t(N) * kPitch;     // [kColGroup][N] the group's columns
    float* snb = reinterpret_cast<float*>(sC + kColGroup * N); // [kColRows]
    __shared__ float2 spro[kColRows / 32][kColGroup]; // prologue sums: warp partials

    for (int idx = tid; idx < kColGroup * N; idx += kColRows) {
        const int c = idx / N, k = idx % N;
        sC[idx] = c < nc ? jb.Y[size_t(n0 + c) * Np + k] : make_float2(0.f, 0.f);
    }
    float nn[kColGroup];
#pragma unroll
    for (int c = 0; c < kColGroup; ++c) nn[c] = c < nc ? jb.nrm[n0 + c] : 0.f;

    const int b_lo = col_begin(n0, capP); // columns of the group start no earlier
    const int b_hi = col_end(n0 + nc - 1, qP, nP);
    // grid.z blocks share a column group, each taking every gridDim.z-th pass of rows
    for (int b0 = b_lo + int(blockIdx.z) * kColRows; b0 < b_hi; b0 += int(gridDim.z) * kColRows) {
        __syncthreads();
        const int nr = min(kColRows, b_hi - b0);
        for (int idx = tid; idx < nr * N; idx += kColRows) {
            const int r = idx / N, k = idx % N;
            sY[k * kPitch + r] = jb.Y[size_t(b0 + r) * Np + k];
        }
        if (tid < nr) snb[tid] = jb.nrm[b0 + tid];
        __syncthreads();
        // sums over the old pairs (pro_range) of every column, for calls that append
        const int pass = (b0 - b_lo) / kColRows;
        const bool pro_any = jb.pro != nullptr;
        float2 pg[kColGroup];
#pragma unroll
        for (int c = 0; c < kColGroup; ++c) pg[c] = make_float2(0.f, 0.f);
        if (tid < nr) {
            const int b = b0 + tid;
            float re[kColGroup], im[kColGroup];
#pragma unroll
            for (int c = 0; c < kColGroup; ++c) re[c] = im[c] = 0.f;
            for (int k = 0; k < N; ++k) {
                const float2 yb = sY[k * kPitch + tid];
#pragma unroll
                for (int c = 0; c < kColGroup; ++c) {
                    const float2 yc = sC[c * N + k];
                    re[c] = fmaf(yb.x, yc.x, fmaf(yb.y, yc.y, re[c]));
                    im[c] = fmaf(yb.x, yc.y, fmaf(-yb.y, yc.x, im[c]));
                }
            }
            const float nb = snb[tid];
#pragma unroll
            for (int c = 0; c < kColGroup; ++c) {
                if (c >= nc) break;
                const int n = n0 + c;
                if (b < col_begin(n, capP) || b >= col_end(n, qP, nP)) continue;
                const float s = nb + nn[c];
                const float A = wG * expf(ew * fmaxf(fmaf(-2.f, re[c], s), 0.f));
                const float Bp = wG * expf(ew * fmaxf(fmaf(-2.f, im[c], s), 0.f));
                const float Bm = wG * expf(ew * fmaxf(fmaf(2.f, im[c], s), 0.f));
                const long long off = column_prefix(n, qP, nP, capP) - jb.kc_base + (b - col_begin(n, capP));
                const float4 kt = make_float4(fmaf(wL, re[c], A), fmaf(wL, im[c], Bp), fmaf(-wL, im[c], Bm), 0.f);
                const_cast<float4*>(jb.Kc)[off] = kt;
                int plo = 0, phi = 0;
                if (pro_any) pro_range(jb, n, &plo, &phi);
                if (b >= plo && b < phi) {
                    // a_2b Kt(2b, .) + a_2b+1 Kt(2b+1, .) for the column pair's two rows
                    const float2 ab = *reinterpret_cast<const float2*>(jb.a + 2 * b);
                    pg[c].x = fmaf(ab.x, kt.x, fmaf(ab.y, kt.z, pg[c].x));
                    pg[c].y = fmaf(ab.x, kt.y, fmaf(ab.y, kt.x, pg[c].y));
                }
            }
        }
        if (pro_any) {
            // this pass's sums: warp shuffles, then the warps in order
#pragma unroll
            for (int c = 0; c < kColGroup; ++c)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    pg[c].x += __shfl_xor_sync(0xffffffffu, pg[c].x, o);
                    pg[c].y += __shfl_xor_sync(0xffffffffu, pg[c].y, o);
                }
            if ((tid & 31) == 0)
#pragma unroll
                for (int c = 0; c < kColGroup; ++c) spro[tid >> 5][c] = pg[c];
            __syncthreads();
            if (tid < nc) {
                float2 v = spro[0][tid];
#pragma unroll
                for (int w = 1; w < kColRows / 32; ++w) {
                    v.x += spro[w][tid].x;
                    v.y += spro[w][tid].y;
                }
                jb.pro[size_t(n0 + tid - jb.n_first) * jb.pro_stride + pass] = v;
            }
        }
    }
}

} // namespace

int batch_kcol_group() { return kColGroup; }
int batch_kcol_rows() { return kColRows; }

cudaError_t launch_batch_kcol(const BatchTrainJob* d_jobs, int n_jobs, int max_cols, int max_n, int row_split,
                              BatchCommon cm, cudaStream_t s)
{
    if (n_jobs <= 0 || max_cols <= 0) return cudaSuccess;
    const size_t smem = sizeof(float2) * (size_t(max_n) * (kColRows + 1) + size_t(kColGroup) * max_n) +
                        sizeof(float) * kColRows;
    cudaError_t e = cudaFuncSetAttribute(batch_kcol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    dim3 grid((max_cols + kColGroup - 1) / kColGroup, n_jobs, row_split > 1 ? row_split : 1);
    batch_kcol_kernel<<<grid, kColRows, smem, s>>>(d_jobs, cm, max_n);
    return cudaGetLastError();
}

} // namespace apsm
