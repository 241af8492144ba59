// Linear least-squares (LLS) detector and the APSM llsInitialization.
//
// Reference: cpp/lib/noma/lls_detector.cu:136-218.  Training solves
//   min_w || A w - y ||,  A = Dedup real rows of the pilots (2P x 2N),
//   y = interleaved (Re, Im) pilot symbols,
// with cuBLAS cublasSgelsBatched (QR, batch 1) exactly as the reference does
// (:163-179); several users are several right-hand sides of one solve.
// Detection is est = A_data w (the reference's cublasSgemm, :207-218), here a
// small kernel over the packed data rows.  llsInitialization copies
// w / linearKernelWeight into the APSM linear weights before training
// (copyWeightMat, cpp/lib/apsm/apsm_noma_detector.cu:321-346).
#include "apsm_host.hpp"
#include "apsm_kernels.cuh"
#include "apsm_lls.cuh"

#include <cublas_v2.h>

#include <string>

namespace apsm {

struct LlsWorkspace {
    cublasHandle_t handle = nullptr;
    DevBuf<float> A, B;
    DevBuf<float*> ptrs; // [A, B] device pointer arrays for the batched call
    DevBuf<float> w;     // users x 2N solution
};

void lls_workspace_free(LlsWorkspace* l)
{
    if (!l) return;
    if (l->handle) cublasDestroy(l->handle);
    delete l;
}

namespace {

// rows (n x Dp, row-major) -> A (n x D, column-major, lda = n)
__global__ void lls_transpose_kernel(const float* __restrict__ rows, int n, int Dp, int D, float* __restrict__ A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * D) return;
    const int r = i % n, d = i / n;
    A[size_t(d) * n + r] = rows[size_t(r) * Dp + d];
}

// y (users x y_stride, rows row0..row0+n) -> B (n x users, column-major)
__global__ void lls_rhs_kernel(const float* __restrict__ y, size_t y_stride, int row0, int n, int users,
                               float* __restrict__ B)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * users) return;
    const int r = i % n, u = i / n;
    B[size_t(u) * n + r] = y[size_t(u) * y_stride + row0 + r];
}

// w[u][d] = B[d + u*n] (the first D rows of each solution column) / divide_by
__global__ void lls_extract_kernel(const float* __restrict__ B, int n, int D, int users, float divide_by,
                                   float* __restrict__ w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D * users) return;
    const int d = i % D, u = i / D;
    const float v = B[size_t(u) * n + d];
    w[size_t(u) * D + d] = divide_by == 1.f ? v : v / divide_by;
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

const char* cublas_msg(cublasStatus_t st)
{
    switch (st) {
    case CUBLAS_STATUS_NOT_INITIALIZED: return "CUBLAS: Not initialized (properly)";
    case CUBLAS_STATUS_ALLOC_FAILED: return "CUBLAS: Allocation failed";
    case CUBLAS_STATUS_INVALID_VALUE: return "CUBLAS: Invalid value";
    case CUBLAS_STATUS_ARCH_MISMATCH: return "CUBLAS: Architecture mismatch";
    case CUBLAS_STATUS_EXECUTION_FAILED: return "CUBLAS: Execution failed";
    case CUBLAS_STATUS_INTERNAL_ERROR: return "CUBLAS: Internal error";
    case CUBLAS_STATUS_NOT_SUPPORTED: return "CUBLAS: Not supported";
    default: return "CUBLAS: Unknown error";
    }
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
    cublasStatus_t cs;
    if (!l->handle) {
        cs = cublasCreate(&l->handle);
        if (cs != CUBLAS_STATUS_SUCCESS) {
            h->last_error = cublas_msg(cs);
            return APSM_ERR_CUDA;
        }
    }
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
    LL_CK(l->A.ensure(size_t(n) * D));
    LL_CK(l->B.ensure(size_t(n) * U));
    LL_CK(l->ptrs.ensure(2));
    LL_CK(l->w.ensure(size_t(U) * D));
    lls_transpose_kernel<<<(n * D + 255) / 256, 256, 0, s>>>(rows, n, int(h->Dp), D, l->A.p);
    LL_CK(cudaGetLastError());
    lls_rhs_kernel<<<(n * U + 255) / 256, 256, 0, s>>>(y, y_stride, row0, n, U, l->B.p);
    LL_CK(cudaGetLastError());
    float* hp[2] = {l->A.p, l->B.p};
    LL_CK(cudaMemcpyAsync(l->ptrs.p, hp, sizeof(hp), cudaMemcpyHostToDevice, s));
    cs = cublasSetStream(l->handle, s);
    int info = 0;
    if (cs == CUBLAS_STATUS_SUCCESS)
        cs = cublasSgelsBatched(l->handle, CUBLAS_OP_N, n, D, U, l->ptrs.p, n, l->ptrs.p + 1, n, &info, nullptr, 1);
    if (cs != CUBLAS_STATUS_SUCCESS) {
        h->last_error = cublas_msg(cs);
        return APSM_ERR_CUDA;
    }
    if (info != 0) {
        h->last_error = "cublasSgelsBatched rejected argument " + std::to_string(-info);
        return APSM_ERR_INVALID_ARGUMENT;
    }
    lls_extract_kernel<<<(D * U + 255) / 256, 256, 0, s>>>(l->B.p, n, D, U, divide_by, l->w.p);
    LL_CK(cudaGetLastError());
    LL_CK(cudaStreamSynchronize(s)); // hp is a host local
#undef LL_CK
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
