// Batched FP32 detection in pair form, all detection jobs of a class of
// antenna counts in one launch.
//
// For data sample s (rows 2s, 2s+1) the reference evaluates
// (cpp/lib/apsm/apsm_detect.cu:526-538 linear, :690-808 Gaussian)
//   f_{2s}   = wL <w, x_2s>   + sum_b a_{2b} K(2b, 2s)   + a_{2b+1} K(2b+1, 2s)
//   f_{2s+1} = wL <w, x_2s+1> + sum_b a_{2b} K(2b, 2s+1) + a_{2b+1} K(2b+1, 2s+1)
// Here each (sample, dictionary pair) costs one complex inner product
// y_b^H y_s (4N fma) and three exponentials instead of four distance loops
// and four exponentials.  Summation order differs from the reference; the
// FP32 bar is 1e-4 relative.
//
// Order of the Gaussian sum: the dictionary is cut into chunks of kChunk
// pairs; each chunk's sum starts from zero and runs over its pairs in order,
// and the chunk sums are added in chunk order.  A launch may give one tile of
// samples to several blocks (grid.z "parts", for batches too small to fill
// the GPU, i.e. single requests): each block then stores its chunk sums
// ([chunk][sample], coalesced) and the tile's last block to arrive adds them
// in chunk order -- the same additions as one block doing every chunk, so the
// estimates do not depend on how a batch was split.
#include "apsm_batch.cuh"

namespace apsm {

namespace {

constexpr int kDetThreads = 128; // samples per block
constexpr int kChunk = 64;       // dictionary pairs per chunk (= one shared-memory tile)
constexpr float kLog2e = 1.4426950408889634f;

template <int NMAX>
__global__ void __launch_bounds__(kDetThreads) batch_detect_kernel(const BatchDetectJob* __restrict__ jobs, float wL,
                                                                   float wG)
{
    const BatchDetectJob& jb = jobs[blockIdx.y];
    const int s0 = blockIdx.x * kDetThreads;
    if (s0 >= jb.S || jb.N > NMAX) return;
    const int N = jb.N, Np = jb.Np, Mp = jb.Mp;
    const int n_chunks = (Mp + kChunk - 1) / kChunk;
    // this block's chunks: runs of cpb chunks, parts_j runs for this job
    const int cpb = n_chunks > 0 ? (n_chunks + int(gridDim.z) - 1) / int(gridDim.z) : 1;
    const int parts_j = n_chunks > 0 ? (n_chunks + cpb - 1) / cpb : 1;
    const int p = blockIdx.z;
    if (p >= parts_j) return;
    const bool split = parts_j > 1;
    const int c_begin = p * cpb, c_end = min(n_chunks, c_begin + cpb);

    const int s = s0 + threadIdx.x;
    const bool valid = s < jb.S;
    const float ew2 = jb.ew * kLog2e;

    __shared__ float2 sD[NMAX][kChunk];
    __shared__ float4 sA[kChunk]; // (a_2b wG, a_2b+1 wG, n_b, 0)
    __shared__ int s_last;

    // the sample straight from the antenna-major input (coalesced per antenna) and its squared
    // norm, real parts first (the order of the training rows' norms)
    float2 ys[NMAX];
#pragma unroll
    for (int k = 0; k < NMAX; ++k) ys[k] = (valid && k < N) ? jb.rx[size_t(k) * jb.S + s] : make_float2(0.f, 0.f);
    float ns = 0.f;
#pragma unroll
    for (int k = 0; k < NMAX; ++k)
        if (k < N) ns = fmaf(ys[k].x, ys[k].x, ns);
#pragma unroll
    for (int k = 0; k < NMAX; ++k)
        if (k < N) ns = fmaf(ys[k].y, ys[k].y, ns);
    float t0 = 0.f, t1 = 0.f; // running sum of the chunk sums (unsplit launches)
    for (int c = c_begin; c < c_end; ++c) {
        const int b0 = c * kChunk;
        const int nb = min(kChunk, Mp - b0);
        __syncthreads();
        for (int idx = threadIdx.x; idx < nb * N; idx += kDetThreads) {
            const int r = idx / N, k = idx % N;
            sD[k][r] = jb.Yd[size_t(b0 + r) * Np + k];
        }
        for (int r = threadIdx.x; r < nb; r += kDetThreads) {
            const float2 ab = *reinterpret_cast<const float2*>(jb.a + 2 * (b0 + r));
            sA[r] = make_float4(ab.x * wG, ab.y * wG, jb.nrm_d[b0 + r], 0.f);
        }
        __syncthreads();
        float f0 = 0.f, f1 = 0.f;
        for (int r = 0; r < nb; ++r) {
            float re = 0.f, im = 0.f;
#pragma unroll
            for (int k = 0; k < NMAX; ++k) {
                if (k < N) {
                    const float2 yb = sD[k][r];
                    re = fmaf(yb.x, ys[k].x, fmaf(yb.y, ys[k].y, re));
                    im = fmaf(yb.x, ys[k].y, fmaf(-yb.y, ys[k].x, im));
                }
            }
            const float4 cf = sA[r];
            const float sum = ns + cf.z;
            const float kA = exp2f(ew2 * fmaxf(fmaf(-2.f, re, sum), 0.f));
            const float kP = exp2f(ew2 * fmaxf(fmaf(-2.f, im, sum), 0.f)); // K(2b, 2s+1)
            const float kM = exp2f(ew2 * fmaxf(fmaf(2.f, im, sum), 0.f));  // K(2b+1, 2s)
            f0 = fmaf(cf.x, kA, fmaf(cf.y, kM, f0));
            f1 = fmaf(cf.x, kP, fmaf(cf.y, kA, f1));
        }
        if (split) {
            if (valid) jb.part[size_t(c) * jb.S + s] = make_float2(f0, f1);
        } else {
            t0 += f0;
            t1 += f1;
        }
    }
    if (split) {
        // the tile's last block adds the chunk sums of all parts in chunk order
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) s_last = atomicAdd(jb.cnt + blockIdx.x, 1) == parts_j - 1;
        __syncthreads();
        if (!s_last) return;
        __threadfence();
        if (valid)
            for (int c = 0; c < n_chunks; ++c) {
                const float2 v = __ldcg(jb.part + size_t(c) * jb.S + s);
                t0 += v.x;
                t1 += v.y;
            }
    }
    float l0 = 0.f, l1 = 0.f;
#pragma unroll
    for (int k = 0; k < NMAX; ++k)
        if (k < N) {
            const float w0 = __ldg(jb.w + k), w1 = __ldg(jb.w + N + k);
            l0 = fmaf(w0, ys[k].x, fmaf(w1, ys[k].y, l0));
            l1 = fmaf(w0, ys[k].y, fmaf(-w1, ys[k].x, l1));
        }
    if (valid) jb.out[s] = make_float2(fmaf(wL, l0, t0), fmaf(wL, l1, t1));
}

} // namespace

cudaError_t launch_batch_detect(const BatchDetectJob* d_jobs, int n_jobs, int max_tiles, int parts, int nmax, float wL,
                                float wG, cudaStream_t s)
{
    if (n_jobs <= 0 || max_tiles <= 0) return cudaSuccess;
    dim3 grid(max_tiles, n_jobs, parts > 1 ? parts : 1);
    switch (nmax) {
    case 4: batch_detect_kernel<4><<<grid, kDetThreads, 0, s>>>(d_jobs, wL, wG); break;
    case 8: batch_detect_kernel<8><<<grid, kDetThreads, 0, s>>>(d_jobs, wL, wG); break;
    case 16: batch_detect_kernel<16><<<grid, kDetThreads, 0, s>>>(d_jobs, wL, wG); break;
    case 32: batch_detect_kernel<32><<<grid, kDetThreads, 0, s>>>(d_jobs, wL, wG); break;
    case 64: batch_detect_kernel<64><<<grid, kDetThreads, 0, s>>>(d_jobs, wL, wG); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int batch_detect_tile() { return kDetThreads; }
int batch_detect_chunk() { return kChunk; }

} // namespace apsm
