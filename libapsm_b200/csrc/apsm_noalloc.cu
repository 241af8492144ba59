// Allocation-free detection (apsm_detect_device_noalloc of include/apsm_b200.h).
//
// apsm_detect_device packs the S data symbols into 2S Dedup rows in a device
// buffer of the handle that grows with S (cudaMalloc on growth).  This entry
// point runs the same two kernels -- pack_rows_kernel, then the exact FP32
// detection in the reference's BALANCED order -- with the packed rows in a
// fixed file-scope device array instead, so the call itself never allocates.
//
// Limits and rules:
//   * the scratch holds kNoAllocScratchBytes (8 MiB): 2 S Dp 4 bytes must fit
//     (Dp = 2N rounded up to 4), e.g. S <= 32768 symbols at N = 16 and
//     S <= 8192 at N = 64; larger S is rejected with APSM_ERR_INVALID_ARGUMENT;
//   * only the exact detection path (the reference's four detectVersion
//     names) of an APSM handle; other handles get APSM_ERR_UNSUPPORTED;
//   * the array's device address is looked up once per device, by the first
//     call on that device, with the handle's device current; make that first
//     call before any stream capture.  The address is kept for the life of
//     the process: cudaDeviceReset of such a device is not supported (the
//     module would be loaded again, possibly at another address);
//   * nothing in the scratch must start at zero: pack_rows_kernel writes every
//     element of every packed row (padding columns included) before the
//     detection kernel reads it;
//   * there is one scratch array per device: calls that overlap on a device
//     (other streams or host threads) race on it and must be serialised by
//     the caller.
#include "apsm_host.hpp"
#include "apsm_kernels.cuh"

#include <mutex>
#include <string>

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_noalloc_rows[kNoAllocScratchBytes / sizeof(float)];

std::mutex g_setup_mu;
float* g_scratch[kMaxDevices] = {};

// Device address of the scratch array on `device` (looked up once per device).
cudaError_t scratch_for(int device, float** out)
{
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(g_setup_mu);
    if (!g_scratch[device]) {
        int prev = -1;
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) return e;
        if (prev != device && (e = cudaSetDevice(device)) != cudaSuccess) return e;
        float* ptr = nullptr;
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_noalloc_rows);
        if (prev != device) cudaSetDevice(prev);
        if (e != cudaSuccess) return e;
        g_scratch[device] = ptr;
    }
    *out = g_scratch[device];
    return cudaSuccess;
}

} // namespace

extern "C" apsm_status apsm_detect_device_noalloc(apsm_detector* h, const float* d_rx, uint32_t S, float* d_est,
                                                  void* stream)
{
    using namespace apsm;
    if (!h) return APSM_ERR_INVALID_ARGUMENT;
    if (!d_rx || !d_est) {
        h->last_error = "detect: null buffer";
        return APSM_ERR_INVALID_ARGUMENT;
    }
    if (h->is_lls || h->cfg.detect_mode != DetectMode::Exact) {
        h->last_error = "allocation-free detection runs the exact FP32 path of an APSM detector only";
        return APSM_ERR_UNSUPPORTED;
    }
    if (S == 0) return APSM_OK;
    const size_t need = sizeof(float) * size_t(2) * S * h->Dp;
    if (need > kNoAllocScratchBytes) {
        h->last_error = "allocation-free detection: " + std::to_string(S) + " symbols need " + std::to_string(need) +
                        " bytes of packed rows, the fixed scratch holds " + std::to_string(kNoAllocScratchBytes);
        return APSM_ERR_INVALID_ARGUMENT;
    }
    float* rows = nullptr;
    cudaError_t e = scratch_for(h->device, &rows);
    if (e != cudaSuccess) return h->cuda_fail(e, "cudaGetSymbolAddress(allocation-free scratch)");
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : h->stream;

    dim3 grid((S + kPackSamples - 1) / kPackSamples);
    pack_rows_kernel<<<grid, 256, sizeof(float2) * h->N * kPackSamples, s>>>(
        reinterpret_cast<const float2*>(d_rx), int(h->N), int(S), nullptr, rows, int(h->Dp), 0, nullptr);
    e = cudaGetLastError();
    if (e != cudaSuccess) return h->cuda_fail(e, "pack_rows_kernel");
    DetectArgs da;
    da.Xs = rows;
    da.n_samples = int(2 * S);
    da.Dp = int(h->Dp);
    da.D = int(h->D);
    da.dict = h->dict_X.p;
    da.M = int(h->used);
    da.a = h->dict_a.p;
    da.a_stride = h->cap;
    da.w = h->w.p;
    da.users = int(h->U);
    da.mp = h->model_params();
    da.out = d_est;
    da.out_stride = size_t(2) * S;
    launch_detect_exact(da, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return h->cuda_fail(e, "detect_exact_kernel");
    return APSM_OK;
}
