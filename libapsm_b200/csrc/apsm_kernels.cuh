// Kernel declarations and launch-argument structs of the B200 APSM library.
#pragma once

#include "apsm_b200.h"
#include "apsm_common.cuh"

#include <string>

namespace apsm {

constexpr int kPackSamples = 64;     // complex samples per pack_rows_kernel block
constexpr int kGramColsPerBlock = 8; // kernel columns per gram_columns_kernel block
constexpr int kGramRows = 128;       // column entries per gram_columns_kernel block (its thread count)
constexpr int kLookahead = 2;        // training steps fetched ahead by cp.async

// First universe row stored in kernel column v (16-byte aligned).
__host__ __device__ inline int column_base(int v, int cap)
{
    const int lo = v + 1 - cap;
    return lo > 0 ? (lo & ~3) : 0;
}

struct TrainArgs {
    const float* X;         // universe rows nU x Dp (old dictionary rows, then the new pilots)
    const float* nrm;       // nU squared row norms
    const float* y;         // users x y_stride targets
    float* a;               // users x a_stride coefficients (in: old rows; out: visible rows)
    float* w;               // users x D linear weights (in/out)
    const float* K;         // nV x Lk kernel columns (gram_columns_kernel), column v starts at row column_base(v)
    const TrainStep* steps; // n_steps
    int n_steps;
    int nU, D, Dp, cap, q2, Lk, v_first;
    int A_ring, XW;         // power-of-two ring sizes (coefficients, window rows)
    int NS, Lc;             // staged kernel columns per CTA and their length (floats)
    int XP;                 // shared-memory pitch of window rows (floats, Dp + 4)
    int XS;                 // window slots of the incremental sweep (row r in slot r % XS)
    int NSO, NSOp;          // incremental sweep: owned-column slots per CTA and their padded pitch
    int used_before;        // rows present before this call
    int final_hi;           // visible end after the last step
    size_t y_stride, a_stride;
    int users;
    ModelParams mp;
    unsigned long long* prof; // phase timestamps (profiling builds only), kProfSteps x kProfMarks
    int* err;                 // set to 1 when a bounded wait expired
    float* snap_a;            // users x n_steps x q2: the active rows' coefficients after each step (nullptr: off)
    float* snap_w;            // users x n_steps x D: the linear weights after each step
    float* snap_scale;        // users x n_steps: the normConstraint factor of each step (1: none)
    float norm_c;             // normConstraint: bound of ||f_G|| after every step (0: off; exact sweep only)
    float* a_glob;            // exact sweep: per-CTA coefficient rings in global memory (nullptr: shared memory)
};

// Training history (kernels_history.cu): every step's model evaluated on the
// call's training rows and a validation set after the sweep.
struct HistoryArgs {
    const TrainStep* steps; // n_steps (the sweep's schedule)
    int n_steps;
    const float* snap_a;    // users x n_steps x q2: active-row coefficients after each step
    const float* snap_w;    // users x n_steps x D: linear weights after each step
    const float* snap_scale; // users x n_steps: normConstraint factor of each step (nullptr: none)
    const float* a0;        // users x a0_stride: coefficients of the rows present before the call
    size_t a0_stride;
    int used_before, nU, cap, q2, D, Dp, users;
    float* A;               // users x n_steps x nU: dense coefficients of every step
    const float* X;         // universe rows nU x Dp
    const float* E;         // evaluation rows nE x Dp: the call's training rows, then the validation rows
    const float* Ey;        // users x nE targets of the evaluation rows
    int nE, n_train;        // evaluation rows (even), of which the first n_train are training rows
    ModelParams mp;
    int bps;                // bits per symbol of the modulation
    float mod_scale;        // constellation scale (unit energy)
    float rev_scale;        // float(1 / scale), as the reference passes it
    float max_val;          // outermost constellation coordinate ((2^(bps/2) - 1) scale)
    int n_tiles;            // evaluation-row tiles
    float* part;            // users x n_steps x n_tiles x 6 partial sums
    float* out;             // users x n_steps x 6: train EVM, SER, BER, validation EVM, SER, BER
};

size_t history_eval_smem(int D);
int history_tiles(int nE);
cudaError_t launch_history(const HistoryArgs& h, cudaStream_t s);

// ApsmNomaDetector::computeNormRatio (kernels_norm_ratio.cu): out[0] = wL |w|^2 / (wG a^T K a)
// over the M dictionary rows X (pitch Dp); row_sums: M floats of scratch.
cudaError_t launch_norm_ratio(const float* X, int Dp, int D, int M, const float* a, const float* w, float ew, float wL,
                              float wG, float* row_sums, float* out, cudaStream_t s);

// computeGaussianVarianceHeuristic on the GPU (kernels_variance.cu): rx N x P antenna-major
// on the device; scratch d_nd of P (P - 1) / 2 floats and d_hist of 256 counters.
apsm_status variance_heuristic_gpu(const float2* d_rx, uint32_t N, uint32_t P, float* d_nd,
                                   unsigned long long* d_hist, cudaStream_t s, float* variance, std::string* err);

constexpr int kProfSteps = 4096;
constexpr int kProfMarks = 8;

__global__ void pack_rows_kernel(const float2* __restrict__ rx, int num_ant, int n_total, const int* __restrict__ perm,
                                 float* __restrict__ X, int Dp, int row0, float* __restrict__ nrm);

__global__ void gather_targets_kernel(const float2* __restrict__ tx, int P, int users, const int* __restrict__ perm,
                                      float* __restrict__ y, size_t y_stride, int row0);

__global__ void gram_columns_kernel(const float* __restrict__ X, int Dp, int D, int nU, int v_first, int nV, int Lk,
                                    int cap, ModelParams mp, float* __restrict__ K);

// Persistent training sweep: one cluster of `cluster` CTAs per user.  Sets
// *max_clusters to the number of clusters that fit the device; launches only
// when that is >= 1.
cudaError_t launch_train_exact(bool staged, int cluster, int threads, size_t smem, cudaStream_t stream,
                               const TrainArgs& args, int* max_clusters);
// Clusters of this shape that fit the device at once.
cudaError_t query_train_clusters(bool staged, bool glob_a, int cluster, int threads, size_t smem, int users,
                                 int* max_clusters);

// Incremental sweep (kernels_sweep_inc.cu): one cluster of `cluster` CTAs per user.
int incremental_threads();
cudaError_t query_incremental_clusters(int cluster, size_t smem, int users, int* max_clusters);
size_t incremental_smem_bytes(int XS, int XP, int NSOp, int A_ring);
cudaError_t launch_train_incremental(int cluster, size_t smem, cudaStream_t stream, const TrainArgs& args,
                                     int* max_clusters);

struct DetectArgs {
    const float* Xs;   // n_samples x Dp data rows (Dedup columns of the received data)
    int n_samples;     // 2S
    int Dp, D;
    const float* dict; // M x Dp dictionary rows
    int M;
    const float* a;    // users x a_stride
    size_t a_stride;
    const float* w;    // users x D
    int users;
    ModelParams mp;
    float* out;        // users x out_stride soft outputs (real rows; complex64 interleaved per symbol)
    size_t out_stride;
};

// Exact FP32 detection in the reference BALANCED kernel's evaluation order.
void launch_detect_exact(const DetectArgs& args, cudaStream_t stream);

} // namespace apsm
