// Batched packing and dictionary copies (one launch for all jobs of a batch).
//
// Packing follows CudaHostMatrix(stream, ComplexSampleMatrix)
// (cpp/lib/cuda/cuda_matrix_host.cu:105-149) but keeps complex samples: pair
// i of the destination is the complex vector (rx[0][p(i)], ..., rx[N-1][p(i)])
// with p the training shuffle (noma_detector.cu:59-74) or the identity.  The
// squared norm is the sequential fma chain over the Dedup row [Re y; Im y],
// the order the single-detector kernels use.
#include "apsm_batch.cuh"

#include <algorithm>

namespace apsm {

namespace {

constexpr int kPackChunk = 64;

// Units (job, chunk of kPackChunk pairs) of a gx-wide grid over the jobs; a block takes units
// blockIdx.x, + gridDim.x, ... (a bounded grid leaves the SMs to concurrent work while the pack
// waits on reads over the host link)
__global__ void __launch_bounds__(256) batch_pack_kernel(const BatchPackJob* __restrict__ jobs, int n_jobs, int gx,
                                                          int smem_n)
{
    extern __shared__ float2 sm[]; // [kPackChunk][N + 1]
    const long long units = (long long)n_jobs * gx;
    for (long long u = blockIdx.x; u < units; u += gridDim.x) {
        const BatchPackJob jb = jobs[u / gx];
        const int i0 = int(u % gx) * kPackChunk;
        if (i0 >= jb.L || jb.N > smem_n) continue; // shared memory is sized for smem_n antennas
        const int n = min(kPackChunk, jb.L - i0);
        const int N = jb.N, Np = jb.Np, pitch = N + 1;
        __syncthreads(); // the previous unit's reads of sm are done
        for (int idx = threadIdx.x; idx < N * kPackChunk; idx += blockDim.x) {
            const int k = idx / kPackChunk, i = idx % kPackChunk;
            if (i < n) {
                const int src = jb.perm ? jb.perm[i0 + i] : i0 + i;
                sm[i * pitch + k] = jb.rx[size_t(k) * jb.L + src];
            }
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < n * Np; idx += blockDim.x) {
            const int i = idx / Np, k = idx % Np;
            jb.Y[size_t(i0 + i) * Np + k] = k < N ? sm[i * pitch + k] : make_float2(0.f, 0.f);
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            float s = 0.f;
            for (int k = 0; k < N; ++k) s = fmaf(sm[i * pitch + k].x, sm[i * pitch + k].x, s);
            for (int k = 0; k < N; ++k) s = fmaf(sm[i * pitch + k].y, sm[i * pitch + k].y, s);
            jb.nrm[i0 + i] = s;
            if (jb.y) {
                const int src = jb.perm ? jb.perm[i0 + i] : i0 + i;
                const float2 t = jb.tx[src];
                jb.y[2 * (i0 + i)] = t.x;
                jb.y[2 * (i0 + i) + 1] = t.y;
            }
            if (jb.a) {
                jb.a[2 * (i0 + i)] = 0.f;
                jb.a[2 * (i0 + i) + 1] = 0.f;
            }
        }
    }
}

__global__ void __launch_bounds__(256) batch_copy_kernel(const BatchCopyJob* __restrict__ jobs)
{
    const BatchCopyJob jb = jobs[blockIdx.y];
    const size_t nY = size_t(jb.pairs) * jb.Np;
    const size_t stride = size_t(gridDim.x) * blockDim.x;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nY; i += stride) jb.Ydst[i] = jb.Ysrc[i];
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < size_t(jb.pairs); i += stride) {
        jb.ndst[i] = jb.nsrc[i];
        jb.ydst[2 * i] = jb.ysrc[2 * i];
        jb.ydst[2 * i + 1] = jb.ysrc[2 * i + 1];
        jb.adst[2 * i] = jb.asrc[2 * i];
        jb.adst[2 * i + 1] = jb.asrc[2 * i + 1];
    }
}

} // namespace

cudaError_t launch_batch_pack(const BatchPackJob* d_jobs, int n_jobs, int max_len, int max_n, cudaStream_t s,
                              int max_blocks)
{
    if (n_jobs <= 0 || max_len <= 0) return cudaSuccess;
    const int gx = (max_len + kPackChunk - 1) / kPackChunk;
    long long blocks = (long long)gx * n_jobs;
    if (max_blocks > 0) blocks = std::min<long long>(blocks, max_blocks);
    batch_pack_kernel<<<unsigned(blocks), 256, sizeof(float2) * kPackChunk * (max_n + 1), s>>>(d_jobs, n_jobs, gx,
                                                                                               max_n);
    return cudaGetLastError();
}

cudaError_t launch_batch_copy(const BatchCopyJob* d_jobs, int n_jobs, int max_pairs, int max_np, cudaStream_t s)
{
    if (n_jobs <= 0 || max_pairs <= 0) return cudaSuccess;
    const long long work = (long long)max_pairs * max_np;
    const int gx = int(std::min<long long>(256, (work + 1023) / 1024));
    batch_copy_kernel<<<dim3(std::max(1, gx), n_jobs), 256, 0, s>>>(d_jobs);
    return cudaGetLastError();
}

} // namespace apsm

namespace apsm {

namespace {

// rows 2b = [Re y_b; Im y_b], 2b+1 = [Im y_b; -Re y_b] of pair b (Dedup embedding,
// cpp/lib/cuda/cuda_matrix_device.cuh:180-188), feature d < Dp (0 past 2N)
__device__ __forceinline__ float dedup_feature(const float2* __restrict__ yb, int N, int odd, int d)
{
    if (d < N) return odd ? yb[d].y : yb[d].x;
    if (d < 2 * N) return odd ? -yb[d - N].x : yb[d - N].y;
    return 0.f;
}

__global__ void pool_to_rows_kernel(const float2* __restrict__ Y, int Np, const float* __restrict__ y,
                                    const float* __restrict__ a, int rows, int N, int Dp, float* __restrict__ X,
                                    float* __restrict__ nrm, float* __restrict__ dy, float* __restrict__ da)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
        const float2* yb = Y + size_t(i >> 1) * Np;
        const int odd = i & 1;
        float acc = 0.f;
        for (int d = 0; d < Dp; ++d) {
            const float v = dedup_feature(yb, N, odd, d);
            X[size_t(i) * Dp + d] = v;
            if (d < 2 * N) acc = fmaf(v, v, acc); // the packing kernels' sequential chain
        }
        nrm[i] = acc;
        dy[i] = y[i];
        da[i] = a[i];
    }
}

__global__ void rows_to_pool_kernel(const float* __restrict__ X, const float* __restrict__ nrm,
                                    const float* __restrict__ dy, const float* __restrict__ da, int rows, int N,
                                    int Dp, int Np, float2* __restrict__ Y, float* __restrict__ pn,
                                    float* __restrict__ y, float* __restrict__ a)
{
    const int pairs = rows / 2;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < pairs; b += gridDim.x * blockDim.x) {
        const float* x = X + size_t(2 * b) * Dp; // row 2b = [Re y_b; Im y_b]
        for (int k = 0; k < Np; ++k) Y[size_t(b) * Np + k] = k < N ? make_float2(x[k], x[N + k]) : make_float2(0.f, 0.f);
        pn[b] = nrm[2 * b]; // the pair norm is row 2b's (same chain: real parts, then imaginary parts)
        y[2 * b] = dy[2 * b];
        y[2 * b + 1] = dy[2 * b + 1];
        a[2 * b] = da[2 * b];
        a[2 * b + 1] = da[2 * b + 1];
    }
}

} // namespace

cudaError_t launch_pool_to_rows(const float2* Y, int Np, const float* y, const float* a, int rows, int N, int Dp,
                                float* X, float* nrm, float* dy, float* da, cudaStream_t s)
{
    if (rows <= 0) return cudaSuccess;
    pool_to_rows_kernel<<<(rows + 127) / 128, 128, 0, s>>>(Y, Np, y, a, rows, N, Dp, X, nrm, dy, da);
    return cudaGetLastError();
}

cudaError_t launch_rows_to_pool(const float* X, const float* nrm, const float* dy, const float* da, int rows, int N,
                                int Dp, int Np, float2* Y, float* pn, float* y, float* a, cudaStream_t s)
{
    if (rows <= 0) return cudaSuccess;
    rows_to_pool_kernel<<<(rows / 2 + 127) / 128, 128, 0, s>>>(X, nrm, dy, da, rows, N, Dp, Np, Y, pn, y, a);
    return cudaGetLastError();
}

} // namespace apsm
