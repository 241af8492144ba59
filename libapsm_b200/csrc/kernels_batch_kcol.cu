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

constexpr int kColGroup = 8;   // columns per block
constexpr int kColRows = 128;  // column entries per block pass (= threads)

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

    for (int idx = tid; idx < kColGroup * N; idx += kColRows) {
        const int c = idx / N, k = idx % N;
        sC[idx] = c < nc ? jb.Y[size_t(n0 + c) * Np + k] : make_float2(0.f, 0.f);
    }
    float nn[kColGroup];
#pragma unroll
    for (int c = 0; c < kColGroup; ++c) nn[c] = c < nc ? jb.nrm[n0 + c] : 0.f;

    const int b_lo = col_begin(n0, capP); // columns of the group start no earlier
    const int b_hi = col_end(n0 + nc - 1, qP, nP);
    for (int b0 = b_lo; b0 < b_hi; b0 += kColRows) {
        __syncthreads();
        const int nr = min(kColRows, b_hi - b0);
        for (int idx = tid; idx < nr * N; idx += kColRows) {
            const int r = idx / N, k = idx % N;
            sY[k * kPitch + r] = jb.Y[size_t(b0 + r) * Np + k];
        }
        if (tid < nr) snb[tid] = jb.nrm[b0 + tid];
        __syncthreads();
        if (tid >= nr) continue;
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
            const_cast<float4*>(jb.Kc)[off] = make_float4(fmaf(wL, re[c], A), fmaf(wL, im[c], Bp), fmaf(-wL, im[c], Bm), 0.f);
        }
    }
}

} // namespace

cudaError_t launch_batch_kcol(const BatchTrainJob* d_jobs, int n_jobs, int max_cols, int max_n, BatchCommon cm,
                              cudaStream_t s)
{
    if (n_jobs <= 0 || max_cols <= 0) return cudaSuccess;
    const size_t smem = sizeof(float2) * (size_t(max_n) * (kColRows + 1) + size_t(kColGroup) * max_n) +
                        sizeof(float) * kColRows;
    cudaError_t e = cudaFuncSetAttribute(batch_kcol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    dim3 grid((max_cols + kColGroup - 1) / kColGroup, n_jobs);
    batch_kcol_kernel<<<grid, kColRows, smem, s>>>(d_jobs, cm, max_n);
    return cudaGetLastError();
}

} // namespace apsm
