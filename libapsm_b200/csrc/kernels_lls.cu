// Linear least-squares (LLS) detector and the APSM llsInitialization.
//
// Reference: cpp/lib/noma/lls_detector.cu:136-218.  Training solves
//   min_w || A w - y ||,  A = Dedup real rows of the pilots (2P x 2N),
//   y = interleaved (Re, Im) pilot symbols,
// which the reference hands to cuBLAS (cublasSgelsBatched, FP32 Householder
// QR, :163-179).  Here the solve runs in this file's kernels, in double
// precision through the normal equations: the Gram matrix A^T A and the
// right-hand sides A^T y are summed over blocks of 64 rows (each block's
// partial in FP64, the blocks added in a fixed order), then one CTA factors
// A^T A = L L^T (Cholesky, in shared memory) and solves for every user.  With
// FP64 the squared condition number costs nothing at these sizes (2N <= 128
// features, kappa(A)^2 * 1e-16 far below FP32 rounding), so the weights are
// the exact least-squares solution rounded to FP32 -- at least as accurate as
// the reference's FP32 QR.  Several users are several right-hand sides of one
// solve.  Detection is est = A_data w (the reference's cublasSgemm,
// :207-218), a small kernel over the packed data rows.  llsInitialization
// copies w / linearKernelWeight into the APSM linear weights before training
// (copyWeightMat, cpp/lib/apsm/apsm_noma_detector.cu:321-346).
#include "apsm_host.hpp"
#include "apsm_kernels.cuh"
#include "apsm_lls.cuh"

#include <string>

namespace apsm {

struct LlsWorkspace {
    DevBuf<double> part; // [blocks][D][D + users] per-block sums (upper triangle of A^T A, then A^T y)
    DevBuf<int> err;     // set when A^T A is not positive definite (rank-deficient pilots)
    DevBuf<float> w;     // users x 2N solution
};

void lls_workspace_free(LlsWorkspace* l) { delete l; }

namespace {

constexpr int kLlsRows = 64;      // pilot rows per Gram block
constexpr int kLlsThreads = 256;
constexpr int kSolveThreads = 1024;

// Per-block sums over rows [blk * kLlsRows, ...): part[blk][i][j] = sum_r x_r[i] z_r[j] with
// z = (features, targets), for j >= i among the features and every target j >= D.
__global__ void __launch_bounds__(kLlsThreads)
    lls_gram_kernel(const float* __restrict__ rows, int n, int Dp, int D, const float* __restrict__ y,
                    size_t y_stride, int row0, int users, double* __restrict__ part)
{
    extern __shared__ float xz[]; // [kLlsRows][D + users]
    const int W = D + users;
    const int r0 = blockIdx.x * kLlsRows;
    const int nr = min(kLlsRows, n - r0);
    for (int idx = threadIdx.x; idx < kLlsRows * W; idx += kLlsThreads) {
        const int r = idx / W, j = idx % W;
        float v = 0.f;
        if (r < nr) v = j < D ? rows[size_t(r0 + r) * Dp + j] : y[size_t(j - D) * y_stride + row0 + r0 + r];
        xz[idx] = v;
    }
    __syncthreads();
    double* out = part + size_t(blockIdx.x) * D * W;
    for (int e = threadIdx.x; e < D * W; e += kLlsThreads) {
        const int i = e / W, j = e % W;
        double acc = 0.0;
        if (j >= i)
            for (int r = 0; r < nr; ++r) acc = fma(double(xz[r * W + i]), double(xz[r * W + j]), acc);
        out[e] = acc;
    }
}

// One CTA: G = sum of the blocks' partials (fixed order), G = L L^T, then
// L L^T w_u = c_u for every user; w[u][d] = w_u[d] / divide_by.
__global__ void __launch_bounds__(kSolveThreads)
    lls_solve_kernel(const double* __restrict__ part, int blocks, int D, int users, float divide_by,
                     float* __restrict__ w, int* __restrict__ err)
{
    extern __shared__ double g[]; // [D][W]: G (lower triangle filled by symmetry) then the right-hand sides
    const int W = D + users;
    __shared__ int bad;
    if (threadIdx.x == 0) bad = 0;
    for (int e = threadIdx.x; e < D * W; e += kSolveThreads) {
        const int i = e / W, j = e % W;
        const int src = (j < D && j < i) ? j * W + i : e; // the upper triangle holds G(i, j) = G(j, i)
        double acc = 0.0;
        for (int b = 0; b < blocks; ++b) acc += part[size_t(b) * D * W + src];
        g[e] = acc;
    }
    __syncthreads();
    // right-looking Cholesky: after step k, column k below the diagonal holds L(., k)
    for (int k = 0; k < D; ++k) {
        const double dkk = g[k * W + k];
        if (!(dkk > 0.0)) {
            if (threadIdx.x == 0) bad = 1;
            break; // uniform: every thread reads the same value
        }
        const double lkk = sqrt(dkk);
        __syncthreads(); // every thread read g(k, k)
        for (int i = k + 1 + threadIdx.x; i < D; i += kSolveThreads) g[i * W + k] /= lkk;
        if (threadIdx.x == 0) g[k * W + k] = lkk;
        __syncthreads();
        // trailing update of the lower triangle: G(i, j) -= L(i, k) L(j, k), k < j <= i
        const int m = D - k - 1;
        for (int e = threadIdx.x; e < m * m; e += kSolveThreads) {
            const int i = k + 1 + e / m, j = k + 1 + e % m;
            if (j <= i) g[i * W + j] -= g[i * W + k] * g[j * W + k];
        }
        __syncthreads();
    }
    __syncthreads();
    if (bad) {
        if (threadIdx.x == 0) *err = 1;
        return;
    }
    // forward (L z = c) then backward (L^T x = z) substitution, one warp per user
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int u = warp; u < users; u += kSolveThreads / 32) {
        double* c = g + D + u; // column D + u, stride W
        for (int i = 0; i < D; ++i) {
            double acc = 0.0;
            for (int j = lane; j < i; j += 32) acc += g[i * W + j] * c[j * W];
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) c[i * W] = (c[i * W] - acc) / g[i * W + i];
            __syncwarp();
        }
        for (int i = D - 1; i >= 0; --i) {
            double acc = 0.0;
            for (int j = i + 1 + lane; j < D; j += 32) acc += g[j * W + i] * c[j * W];
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) c[i * W] = (c[i * W] - acc) / g[i * W + i];
            __syncwarp();
        }
        for (int d = lane; d < D; d += 32) w[size_t(u) * D + d] = float(c[d * W] / double(divide_by));
    }
}

// out[u][s] = sum_d xs[s][d] * w[u][d]
__global__ void lls_detect_kernel(const float* __restrict__ xs, int ns, int Dp, int D, const float* __restrict__ w,
                                  int users, float* __restrict__ out, size_t out_stride)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ns * users) return;
    const int s = i % ns, u = i / ns;
    float acc = 0.f;
    for (int d = 0; d < D; ++d) acc = fmaf(xs[size_t(s) * Dp + d], w[size_t(u) * D + d], acc);
    out[size_t(u) * out_stride + s] = acc;
}

} // namespace

// Solve for every user's linear weights from the packed pilot rows
// (rows: n = 2P rows of pitch Dp; targets y rows [row0, row0 + n)).
// On success h->lls->w holds users x 2N weights divided by `divide_by`.
apsm_status lls_solve(apsm_detector* h, const float* rows, int n, const float* y, size_t y_stride, int row0,
                      float divide_by, cudaStream_t s)
{
    const int D = int(h->D), U = int(h->U);
    if (!h->lls) h->lls = new LlsWorkspace();
    LlsWorkspace* l = h->lls;
    if (n < D) {
        h->last_error = "LLS needs at least as many real pilot rows as features (2P >= 2N)";
        return APSM_ERR_INVALID_ARGUMENT;
    }
    cudaError_t e;
#define LL_CK(x)                                              \
    do {                                                      \
        e = (x);                                              \
        if (e != cudaSuccess) return h->cuda_fail(e, #x);     \
    } while (0)
    const int W = D + U;
    const int blocks = (n + kLlsRows - 1) / kLlsRows;
    LL_CK(l->part.ensure(size_t(blocks) * D * W));
    LL_CK(l->err.ensure(1));
    LL_CK(l->w.ensure(size_t(U) * D));
    LL_CK(cudaMemsetAsync(l->err.p, 0, sizeof(int), s));
    lls_gram_kernel<<<blocks, kLlsThreads, sizeof(float) * kLlsRows * W, s>>>(rows, n, int(h->Dp), D, y, y_stride,
                                                                             row0, U, l->part.p);
    LL_CK(cudaGetLastError());
    const size_t smem = sizeof(double) * size_t(D) * W;
    if (smem > 227 * 1024) {
        h->last_error = "LLS: " + std::to_string(U) + " users with " + std::to_string(D) +
                        " features exceed the solver's shared memory";
        return APSM_ERR_UNSUPPORTED;
    }
    LL_CK(cudaFuncSetAttribute(lls_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    lls_solve_kernel<<<1, kSolveThreads, smem, s>>>(l->part.p, blocks, D, U, divide_by, l->w.p, l->err.p);
    LL_CK(cudaGetLastError());
    int bad = 0;
    LL_CK(cudaMemcpyAsync(&bad, l->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    LL_CK(cudaStreamSynchronize(s));
#undef LL_CK
    if (bad) {
        h->last_error = "LLS: the pilots' feature matrix is rank-deficient (A^T A not positive definite)";
        return APSM_ERR_INVALID_ARGUMENT;
    }
    return APSM_OK;
}

apsm_status lls_detect(apsm_detector* h, int ns, float* d_out, cudaStream_t s)
{
    if (!h->lls || h->used == 0) {
        // untrained: the reference's weight matrix is uninitialised device memory;
        // here an untrained LLS detector outputs zeros
        cudaError_t e = cudaMemsetAsync(d_out, 0, sizeof(float) * size_t(h->U) * ns, s);
        return e == cudaSuccess ? APSM_OK : h->cuda_fail(e, "cudaMemsetAsync");
    }
    const int U = int(h->U);
    lls_detect_kernel<<<(ns * U + 255) / 256, 256, 0, s>>>(h->xs.p, ns, int(h->Dp), int(h->D), h->lls->w.p, U, d_out,
                                                          size_t(ns));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? APSM_OK : h->cuda_fail(e, "lls_detect_kernel");
}

const float* lls_weights(apsm_detector* h) { return h->lls ? h->lls->w.p : nullptr; }

} // namespace apsm
