/* TEST INFRASTRUCTURE ONLY — the oracle is the checker, never the product.
 *
 * CPU restatement of the reference APSM path (fraunhoferhhi/libapsm):
 *   training  cpp/lib/apsm/apsm_train.cu:80-166 (host step loop) and :271-432 (kernel)
 *   prediction cpp/lib/apsm/apsm_detect.cu:103-226 (device fns used by training)
 *   detection cpp/lib/apsm/apsm_detect.cu:690-876 (BALANCED, the default variant)
 *   Dedup     cpp/lib/cuda/cuda_matrix_device.cuh:180-188, 288-296
 *   window    cpp/lib/cuda/cuda_matrix_host.cu:334-365
 *
 * Two precisions:
 *   APSM_ORACLE_F32  float arithmetic in the reference's evaluation order
 *                    (per-lane partial sums, fma where nvcc contracts, the
 *                    BALANCED warp-shuffle tree in detection).  Also the timed
 *                    CPU baseline (OpenMP over window elements / samples).
 *   APSM_ORACLE_F64  the same model in double precision (accuracy oracle).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 */
#ifndef APSM_ORACLE_H
#define APSM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { APSM_ORACLE_F32 = 0, APSM_ORACLE_F64 = 1 };

/* Parameters exactly as the reference stores them (apsm_parameters.cuh:68-86),
 * i.e. after ApsmNomaDetectorFactory::build and the constructor's N^2 scaling of
 * the variance (apsm_noma_detector.cu:79-80, :348-383). */
typedef struct {
    float linear_weight;
    float gaussian_weight;
    float gaussian_variance; /* effective: JSON value * N^2 */
    float eB;
    uint32_t window_size;
    uint32_t sample_step;
    uint32_t train_passes;
    uint32_t start_full_window;
    uint32_t dictionary_size; /* complex entries; 2x real rows */
    float norm_constraint;    /* > 0: RKHS-norm bound of the Gaussian part, applied after every step */
} apsm_oracle_params;

typedef struct apsm_oracle apsm_oracle;

apsm_oracle* apsm_oracle_create(const apsm_oracle_params* par, uint32_t n_ant, int precision);
void apsm_oracle_destroy(apsm_oracle* o);
void apsm_oracle_reset(apsm_oracle* o);
int apsm_oracle_set_threads(int n);

/* rx: antenna-major complex (re,im) pairs, rx[2*(a*P+n)+{0,1}]; tx: P complex. */
int apsm_oracle_train(apsm_oracle* o, const float* rx, const float* tx, uint32_t P);
/* Training that records the reference's per-step history (NomaTrainHistory,
 * noma_train_history.cu:65-248, apsm_train.cu:147-156): after every step the
 * rows of this call and S validation samples (rx_val antenna-major, tx_val S
 * complex) are detected and history[step * 6 + {0..5}] = train EVM, SER, BER,
 * validation EVM, SER, BER.  F32 oracles only.  *n_steps = steps trained;
 * returns 3 when that exceeds max_steps (the first max_steps are written). */
int apsm_oracle_train_history(apsm_oracle* o, const float* rx, const float* tx, uint32_t P, const float* rx_val,
                              const float* tx_val, uint32_t S, uint32_t bps, float mod_scale, float* history,
                              uint32_t max_steps, uint32_t* n_steps);
/* computeNormRatio of the current model (F32 oracles). */
float apsm_oracle_norm_ratio(const apsm_oracle* o);
/* est: S complex (re,im). */
int apsm_oracle_detect(apsm_oracle* o, const float* rx, uint32_t S, float* est);

/* State access (logical row order, oldest first). Sizes: rows <= 2*dictionary_size. */
uint32_t apsm_oracle_rows(const apsm_oracle* o);
void apsm_oracle_get_state(const apsm_oracle* o, double* dict /*rows x 2N*/, double* y /*rows*/,
                           double* a /*rows*/, double* w /*2N*/);
/* Replace the model (dictionary rows, coefficients, linear weights); targets are set to 0. */
int apsm_oracle_set_state(apsm_oracle* o, uint32_t rows, const double* dict, const double* a, const double* w);

/* Replace the effective Gaussian variance (the reference's heuristic path sets it in train()). */
void apsm_oracle_set_variance(apsm_oracle* o, float variance);

/* Replace the linear weights (llsInitialization, apsm_noma_detector.cu:321-346). */
void apsm_oracle_set_w(apsm_oracle* o, const double* w);

/* trainingShuffle permutation (shuffle.cpp). */
void apsm_oracle_shuffle_permutation(uint32_t P, int32_t* perm);

#ifdef __cplusplus
}
#endif
#endif
