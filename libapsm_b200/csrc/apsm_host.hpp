// Host-side detector object behind the C ABI.
#pragma once

#include "apsm_b200.h"
#include "apsm_common.cuh"

#include <cuda_runtime.h>
#include <string>
#include <vector>

namespace apsm {

enum class DetectMode { Exact, GramBF16, GramBF16x3, GramTF32, GramTF32x3 };

// The reference's apsm_parameters (apsm_parameters.cuh:68-86) plus the
// algorithm selector, as read from the JSON config.
struct Config {
    std::string otype = "APSM";
    bool lls_init = false;
    bool shuffle = false;
    float wG = 0.5f;
    float wL = 0.5f;
    float variance = 0.05f; // JSON value; the detector scales it by N^2
    uint32_t window = 20;
    uint32_t step = 2;
    uint32_t passes = 1;
    bool sfw = false;
    uint32_t dict_size = 685;
    float norm_constraint = 0.f;
    float eB = 0.001f;
    std::string detect_version = "balanced";
    DetectMode detect_mode = DetectMode::Exact;
    bool train_incremental = false; // "trainVersion": "incremental"
};

Config parse_config(const std::string& json_text);
std::vector<TrainStep> build_schedule(const Config& c, uint32_t used_before, uint32_t P, uint32_t cap, int* final_hi);
std::vector<int> shuffle_permutation(uint32_t P);

// Growable device buffer.
template <class T> struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t ensure(size_t count)
    {
        if (count <= n) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            return e;
        }
        n = count;
        return cudaSuccess;
    }
};

// Validation set and output of a training call that records its per-step
// history (device buffers).
struct HistoryRequest {
    const float2* rx_val; // N x S antenna-major
    const float2* tx_val; // users x S
    uint32_t S = 0;
    uint32_t bps = 0;
    float mod_scale = 0.f;
    float* out = nullptr; // users x n_steps x 6
    uint32_t max_steps = 0;
    uint32_t n_steps = 0; // set by train(): steps recorded
};

struct GramWorkspace; // tensor-core detection operands (kernels_detect_gram.cu)
struct LlsWorkspace;  // least-squares solver state (kernels_lls.cu)

} // namespace apsm

struct apsm_detector {
    apsm::Config cfg;
    uint32_t N = 0, D = 0, Dp = 0, U = 1, cap = 0;
    float variance_eff = 0.f; // gaussianKernelVariance after the N^2 scaling
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // stage events of the last train / detect call: [sweep start, sweep end, detect start, detect end]
    cudaEvent_t stage_ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool stage_valid[2] = {false, false};
    std::string last_error;

    // persistent model (dictionary rows oldest first, per-user targets and coefficients)
    uint32_t used = 0;
    apsm::DevBuf<float> dict_X, dict_nrm, dict_y, dict_a, w;

    // per-call scratch
    apsm::DevBuf<float> uX, unrm, uy, ua, K, xs;
    apsm::DevBuf<float> a_rings; // exact sweep: per-CTA coefficient rings of large dictionaries
    apsm::DevBuf<apsm::TrainStep> steps;
    apsm::DevBuf<int> train_err; // set by the sweep when a bounded wait expired
    apsm::DevBuf<int> perm;
    apsm::DevBuf<float2> rx_stage, tx_stage, est_stage;
    // training-history scratch: per-step snapshots, initial coefficients, dense
    // per-step coefficients, evaluation rows / targets, partial sums, output
    apsm::DevBuf<float> h_snap_a, h_snap_w, h_snap_scale, h_a0, h_A, h_E, h_Ey, h_part, h_out;
    apsm::DevBuf<float2> h_rx, h_tx;
    apsm::DevBuf<float> nr_scratch; // norm ratio: row sums and the result
    apsm::DevBuf<float> vh_nd;      // variance heuristic: pair distances
    apsm::DevBuf<unsigned long long> vh_hist;
    apsm::GramWorkspace* gram = nullptr;
    apsm::LlsWorkspace* lls = nullptr; // least-squares detector / llsInitialization
    bool is_lls = false;               // "otype": "LLS"
    bool gram_one_product = false;     // APSM_GRAM_ONE_PRODUCT=1: users' sums on the CUDA cores for any user count

    // training-kernel launch shape: requested cluster size, and the last one used
    int cluster = 0;
    int last_train_cluster = 0;
    bool last_train_staged = false;
    bool last_train_glob_a = false; // the last exact sweep kept its coefficient rings in global memory
    bool force_glob_a = false;      // APSM_TRAIN_GLOBAL_RING=1: global rings for every exact sweep
    unsigned long long* prof_buffer = nullptr; // device timestamps of profiling builds

    ~apsm_detector();
    apsm_status init(const apsm::Config& c, uint32_t num_antennas, uint32_t num_users);
    apsm_status reset();
    apsm_status train(const float2* d_rx, const float2* d_tx, uint32_t P, cudaStream_t s, float* ms,
                      apsm::HistoryRequest* hist = nullptr);
    apsm_status train_history_host(const float2* rx, const float2* tx, uint32_t P, const float2* rx_val,
                                   const float2* tx_val, uint32_t S, uint32_t bps, float mod_scale, float* history,
                                   uint32_t max_steps, uint32_t* n_steps, float* ms);
    uint32_t train_steps(uint32_t P) const;
    apsm_status norm_ratio(uint32_t user, float* ratio);
    float gaussian_variance() const { return variance_eff; }
    apsm_status detect(const float2* d_rx, uint32_t S, float2* d_est, cudaStream_t s);
    apsm_status train_host(const float2* rx, const float2* tx, uint32_t P, float* ms);
    apsm_status detect_host(const float2* rx, uint32_t S, float2* est, float* ms);
    apsm_status get_state(float* dict, float* a, float* w_out);
    apsm_status copy_state_from(const apsm_detector& src);
    apsm_status stage_ms(float* sweep_ms, float* detect_ms);
    apsm_status check_train_error();
    apsm::ModelParams model_params() const;
    apsm_status cuda_fail(cudaError_t e, const char* what);
};
