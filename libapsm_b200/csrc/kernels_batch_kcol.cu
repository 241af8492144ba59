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

__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Block: kColGroup columns (the group's pairs y_n and norms in shared memory,
// read as broadcasts) against passes of kColRows rows, one row per thread held
// in registers (NMAX >= N antennas of every job of the launch).
template <int NMAX>
__global__ void __launch_bounds__(kColRows)
    batch_kcol_kernel(const BatchTrainJob* __restrict__ jobs, const int* __restrict__ order, BatchCommon cm)
{
    // the job's fields in registers: the column stores below cannot alias them then
    const BatchTrainJob& jg = jobs[order ? order[blockIdx.y] : int(blockIdx.y)];
    const int nP = jg.nP, N = jg.N, Np = jg.Np, capP = jg.capP, qP = cm.qP;
    const int n_first = jg.n_first;
    const int n0 = n_first + blockIdx.x * kColGroup;
    if (n0 >= nP || N > NMAX) return;
    const int nc = min(kColGroup, nP - n0);
    const float2* __restrict__ Y = jg.Y;
    const float* __restrict__ nrm = jg.nrm;
    const float* __restrict__ a = jg.a;
    float4* __restrict__ Kc = const_cast<float4*>(jg.Kc);
    float2* __restrict__ pro = jg.pro;
    const int pro_stride = jg.pro_stride;
    // exp(ew x) = 2^(ew log2(e) x) on the SFU
    const float ewl2 = jg.ew * 1.4426950408889634f, wG = cm.wG, wL = cm.wL;
    const int tid = threadIdx.x;

    __shared__ __align__(16) float2 sC[NMAX][kColGroup]; // the group's columns, feature-major
    __shared__ float2 spro[kColRows / 32][kColGroup];      // prologue sums: warp partials
    // per column: entry range [blo, bhi), store offset of entry b (off + b), old-pair range of its sums
    __shared__ long long s_off[kColGroup];
    __shared__ int s_blo[kColGroup], s_bhi[kColGroup], s_plo[kColGroup], s_phi[kColGroup];

    if (tid < kColGroup) {
        const int n = n0 + tid;
        int blo = 0, bhi = 0, plo = 0, phi = 0;
        long long off = 0;
        if (tid < nc) {
            blo = col_begin(n, capP);
            bhi = col_end(n, qP, nP);
            off = column_prefix(n, qP, nP, capP) - jg.kc_base - blo;
            if (pro) pro_range(jg, n, &plo, &phi);
        }
        s_blo[tid] = blo;
        s_bhi[tid] = bhi;
        s_off[tid] = off;
        s_plo[tid] = plo;
        s_phi[tid] = phi;
    }
    for (int idx = tid; idx < kColGroup * N; idx += kColRows) {
        const int k = idx / kColGroup, c = idx % kColGroup;
        sC[k][c] = c < nc ? Y[size_t(n0 + c) * Np + k] : make_float2(0.f, 0.f);
    }
    float nn[kColGroup];
#pragma unroll
    for (int c = 0; c < kColGroup; ++c) nn[c] = c < nc ? nrm[n0 + c] : 0.f;
    __syncthreads();

    const int b_lo = col_begin(n0, capP); // columns of the group start no earlier
    const int b_hi = col_end(n0 + nc - 1, qP, nP);
    // grid.z blocks share a column group, each taking every gridDim.z-th pass of rows
    for (int b0 = b_lo + int(blockIdx.z) * kColRows; b0 < b_hi; b0 += int(gridDim.z) * kColRows) {
        // sums over the old pairs (pro_range) of every column, for calls that append
        const int pass = (b0 - b_lo) / kColRows;
        float2 pg[kColGroup];
#pragma unroll
        for (int c = 0; c < kColGroup; ++c) pg[c] = make_float2(0.f, 0.f);
        const int b = b0 + tid;
        if (b < b_hi) {
            // this thread's row (rows are 16-byte aligned: Np is even)
            float2 yb[NMAX];
            const float4* row = reinterpret_cast<const float4*>(Y + size_t(b) * Np);
#pragma unroll
            for (int j = 0; j < NMAX / 2; ++j) {
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (2 * j < N) v = __ldg(row + j);
                yb[2 * j] = make_float2(v.x, v.y);
                yb[2 * j + 1] = make_float2(v.z, v.w);
            }
            const float nb = __ldg(nrm + b);
            float re[kColGroup], im[kColGroup];
#pragma unroll
            for (int c = 0; c < kColGroup; ++c) re[c] = im[c] = 0.f;
#pragma unroll
            for (int k = 0; k < NMAX; ++k) {
                if (k >= N) break;
                const float4* c4 = reinterpret_cast<const float4*>(&sC[k][0]);
#pragma unroll
                for (int h = 0; h < kColGroup / 2; ++h) {
                    const float4 v = c4[h]; // columns 2h (x, y) and 2h + 1 (z, w)
                    re[2 * h] = fmaf(yb[k].x, v.x, fmaf(yb[k].y, v.y, re[2 * h]));
                    im[2 * h] = fmaf(yb[k].x, v.y, fmaf(-yb[k].y, v.x, im[2 * h]));
                    re[2 * h + 1] = fmaf(yb[k].x, v.z, fmaf(yb[k].y, v.w, re[2 * h + 1]));
                    im[2 * h + 1] = fmaf(yb[k].x, v.w, fmaf(-yb[k].y, v.z, im[2 * h + 1]));
                }
            }
#pragma unroll
            for (int c = 0; c < kColGroup; ++c) {
                if (c >= nc) break;
                if (b < s_blo[c] || b >= s_bhi[c]) continue;
                const float sn = nb + nn[c];
                const float A = wG * ex2_approx(ewl2 * fmaxf(fmaf(-2.f, re[c], sn), 0.f));
                const float Bp = wG * ex2_approx(ewl2 * fmaxf(fmaf(-2.f, im[c], sn), 0.f));
                const float Bm = wG * ex2_approx(ewl2 * fmaxf(fmaf(2.f, im[c], sn), 0.f));
                const float4 kt = make_float4(fmaf(wL, re[c], A), fmaf(wL, im[c], Bp), fmaf(-wL, im[c], Bm), 0.f);
                Kc[s_off[c] + b] = kt;
                if (b >= s_plo[c] && b < s_phi[c]) {
                    // a_2b Kt(2b, .) + a_2b+1 Kt(2b+1, .) for the column pair's two rows
                    const float2 ab = *reinterpret_cast<const float2*>(a + 2 * b);
                    pg[c].x = fmaf(ab.x, kt.x, fmaf(ab.y, kt.z, pg[c].x));
                    pg[c].y = fmaf(ab.x, kt.y, fmaf(ab.y, kt.x, pg[c].y));
                }
            }
        }
        if (pro) {
            // this pass's sums: warp shuffles, then the warps in order
#pragma unroll
            for (int c = 0; c < kColGroup; ++c)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    pg[c].x += __shfl_xor_sync(0xffffffffu, pg[c].x, o);
                    pg[c].y += __shfl_xor_sync(0xffffffffu, pg[c].y, o);
                }
            __syncthreads(); // the previous pass's partials were read
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
                pro[size_t(n0 + tid - n_first) * pro_stride + pass] = v;
            }
        }
    }
}

} // namespace

int batch_kcol_group() { return kColGroup; }
int batch_kcol_rows() { return kColRows; }

cudaError_t launch_batch_kcol(const BatchTrainJob* d_jobs, const int* order, int n_jobs, int max_cols, int max_n,
                              int row_split, BatchCommon cm, cudaStream_t s)
{
    if (n_jobs <= 0 || max_cols <= 0) return cudaSuccess;
    dim3 grid((max_cols + kColGroup - 1) / kColGroup, n_jobs, row_split > 1 ? row_split : 1);
    if (max_n <= 4) batch_kcol_kernel<4><<<grid, kColRows, 0, s>>>(d_jobs, order, cm);
    else if (max_n <= 8) batch_kcol_kernel<8><<<grid, kColRows, 0, s>>>(d_jobs, order, cm);
    else if (max_n <= 16) batch_kcol_kernel<16><<<grid, kColRows, 0, s>>>(d_jobs, order, cm);
    else if (max_n <= 32) batch_kcol_kernel<32><<<grid, kColRows, 0, s>>>(d_jobs, order, cm);
    else if (max_n <= 64) batch_kcol_kernel<64><<<grid, kColRows, 0, s>>>(d_jobs, order, cm);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

} // namespace apsm
