/* TEST INFRASTRUCTURE ONLY — the oracle is the checker, never the product.
 * See apsm_oracle.h for the reference files this restates.
 *
 * Built with -ffp-contract=off: every fused multiply-add below is written as
 * fmaf() exactly where nvcc contracts the reference's expression, every other
 * product and sum rounds separately, as in the reference kernels.
 */
#include "apsm_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#define LANES 32u   /* APSM_BLOCK_BATCH_SIZE / WARP_SIZE (cpp/lib/cuda/cuda_indexing.cuh:74) */
#define WGROUPS 8u  /* linear-weight update: window terms are summed in 8 interleaved groups */

struct apsm_oracle {
    apsm_oracle_params par;
    int prec;
    uint32_t n_ant, D, cap;
    uint32_t used, head; /* ring: logical row r lives in physical row (head + r) % cap */
    float *Xf, *Yf, *Af, *Wf;
    double *Xd, *Yd, *Ad, *Wd;
};

static uint32_t umin(uint32_t a, uint32_t b) { return a < b ? a : b; }
static uint32_t umax(uint32_t a, uint32_t b) { return a > b ? a : b; }

int apsm_oracle_set_threads(int n)
{
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
}

apsm_oracle* apsm_oracle_create(const apsm_oracle_params* par, uint32_t n_ant, int precision)
{
    if (!par || n_ant == 0 || par->dictionary_size == 0) return NULL;
    apsm_oracle* o = (apsm_oracle*)calloc(1, sizeof(apsm_oracle));
    o->par = *par;
    o->prec = precision;
    o->n_ant = n_ant;
    o->D = 2 * n_ant;
    o->cap = 2 * par->dictionary_size; /* HostTrainingState(2N, 2*dictSize), apsm_noma_detector.cu:92 */
    size_t rows = o->cap, D = o->D;
    if (precision == APSM_ORACLE_F32) {
        o->Xf = (float*)calloc(rows * D, sizeof(float));
        o->Yf = (float*)calloc(rows, sizeof(float));
        o->Af = (float*)calloc(rows, sizeof(float));
        o->Wf = (float*)calloc(D, sizeof(float));
    } else {
        o->Xd = (double*)calloc(rows * D, sizeof(double));
        o->Yd = (double*)calloc(rows, sizeof(double));
        o->Ad = (double*)calloc(rows, sizeof(double));
        o->Wd = (double*)calloc(D, sizeof(double));
    }
    return o;
}

void apsm_oracle_destroy(apsm_oracle* o)
{
    if (!o) return;
    free(o->Xf); free(o->Yf); free(o->Af); free(o->Wf);
    free(o->Xd); free(o->Yd); free(o->Ad); free(o->Wd);
    free(o);
}

void apsm_oracle_reset(apsm_oracle* o)
{
    size_t rows = o->cap, D = o->D;
    o->used = 0;
    o->head = 0;
    if (o->prec == APSM_ORACLE_F32) {
        memset(o->Xf, 0, rows * D * sizeof(float));
        memset(o->Yf, 0, rows * sizeof(float));
        memset(o->Af, 0, rows * sizeof(float));
        memset(o->Wf, 0, D * sizeof(float));
    } else {
        memset(o->Xd, 0, rows * D * sizeof(double));
        memset(o->Yd, 0, rows * sizeof(double));
        memset(o->Ad, 0, rows * sizeof(double));
        memset(o->Wd, 0, D * sizeof(double));
    }
}

static uint32_t phys(const apsm_oracle* o, uint32_t r) { return (o->head + r) % o->cap; }

/* Dedup embedding of complex sample n (cuda_matrix_device.cuh:180-188):
 * real column 2n   = [Re y_n ; Im y_n]
 * real column 2n+1 = [Im y_n ; -Re y_n]                                   */
static void dedup_column(const float* rx, uint32_t n_ant, uint32_t n_samp, uint32_t col, float* x)
{
    uint32_t n = col >> 1;
    for (uint32_t a = 0; a < n_ant; ++a) {
        float re = rx[2 * ((size_t)a * n_samp + n)];
        float im = rx[2 * ((size_t)a * n_samp + n) + 1];
        if ((col & 1u) == 0) {
            x[a] = re;
            x[n_ant + a] = im;
        } else {
            x[a] = im;
            x[n_ant + a] = -re;
        }
    }
}

/* Make one more staged row visible (moveWindow by one row, cuda_matrix_host.cu:355-365).
 * When the ring is full the oldest row is evicted and the new row starts with a = 0. */
static void reveal_row(apsm_oracle* o, const float* x, float y)
{
    uint32_t p;
    if (o->used < o->cap) {
        p = phys(o, o->used);
        o->used++;
    } else {
        p = o->head;
        o->head = (o->head + 1) % o->cap;
    }
    for (uint32_t d = 0; d < o->D; ++d) {
        if (o->prec == APSM_ORACLE_F32) o->Xf[(size_t)p * o->D + d] = x[d];
        else o->Xd[(size_t)p * o->D + d] = (double)x[d];
    }
    if (o->prec == APSM_ORACLE_F32) { o->Yf[p] = y; o->Af[p] = 0.f; }
    else { o->Yd[p] = (double)y; o->Ad[p] = 0.0; }
}

/* ---------------------------------------------------------------- FP32 -- */

/* exp(-||d-x||^2 / (2 s^2)) in the reference's order (apsm_detect.cu:131-152):
 * sequential fma over dims, float exp weight -0.5f/variance. */
static float kern_f32(const float* d, const float* x, uint32_t D, float ew)
{
    float acc = 0.f;
    for (uint32_t k = 0; k < D; ++k) {
        float diff = d[k] - x[k];
        acc = fmaf(diff, diff, acc);
    }
    return expf(ew * acc);
}

/* Training prediction f(x_j) (apsm_detect.cu:170-226 + apsm_train.cu:349-356):
 * lane l accumulates basis indices b = l, l+32, ...; each b adds its linear
 * term (b < D) then its Gaussian term (b < used); thread 0 then sums the 32
 * partials sequentially. */
static float predict_train_f32(const apsm_oracle* o, const float* x)
{
    const apsm_oracle_params* p = &o->par;
    const float ew = -0.5f / p->gaussian_variance;
    float part[LANES];
    memset(part, 0, sizeof(part));
    uint32_t L = umax(o->D, o->used);
    for (uint32_t b = 0; b < L; ++b) {
        uint32_t l = b & (LANES - 1);
        if (b < o->D) {
            float ke = p->linear_weight * x[b];
            ke = ke * o->Wf[b];
            part[l] = part[l] + ke;
        }
        if (b < o->used) {
            uint32_t r = phys(o, b);
            float ke = p->gaussian_weight * kern_f32(&o->Xf[(size_t)r * o->D], x, o->D, ew);
            ke = ke * o->Af[r];
            part[l] = part[l] + ke;
        }
    }
    float f = part[0];
    for (uint32_t l = 1; l < LANES; ++l) f = f + part[l];
    return f;
}

/* Hyperslab projection coefficient (apsm_train.cu:380-401). */
static float project_f32(const apsm_oracle* o, float e, uint32_t wk, const float* x)
{
    const apsm_oracle_params* p = &o->par;
    float c = 0.f;
    if (e > p->eB) c = e - p->eB;
    else if (e < -p->eB) c = e + p->eB;
    float lin = 0.f;
    for (uint32_t d = 0; d < o->D; ++d) lin = fmaf(x[d], x[d], lin);
    float linearNorm = p->linear_weight * lin;
    float gaussianNorm = p->gaussian_weight;
    c = c / (float)wk;
    c = c / (linearNorm + gaussianNorm);
    return c;
}

static void step_f32(apsm_oracle* o, uint32_t start, uint32_t n_active, uint32_t wk, float* f, float* c)
{
    const uint32_t D = o->D;
#pragma omp parallel for schedule(static) if (n_active > 8)
    for (uint32_t i = 0; i < n_active; ++i) {
        uint32_t r = phys(o, start + i);
        f[i] = predict_train_f32(o, &o->Xf[(size_t)r * D]);
    }
    for (uint32_t i = 0; i < n_active; ++i) {
        uint32_t r = phys(o, start + i);
        c[i] = project_f32(o, o->Yf[r] - f[i], wk, &o->Xf[(size_t)r * D]);
    }
    /* all predictions used the pre-step coefficients (grid sync, apsm_train.cu:367) */
    for (uint32_t i = 0; i < n_active; ++i) {
        uint32_t r = phys(o, start + i);
        o->Af[r] = o->Af[r] + c[i];
    }
    /* w += sum_j c_j x_j.  The reference adds the terms with float atomics in
     * whatever order the blocks run (apsm_train.cu:425).  The order fixed here
     * (and by the CUDA kernel): 8 groups by window position mod 8, each summed
     * in ascending position, combined as ((g0+g1)+(g2+g3))+((g4+g5)+(g6+g7)). */
    for (uint32_t d = 0; d < D; ++d) {
        float g[WGROUPS];
        memset(g, 0, sizeof(g));
        for (uint32_t i = 0; i < n_active; ++i) {
            if (c[i] == 0.f) continue;
            uint32_t r = phys(o, start + i);
            float t = c[i] * o->Xf[(size_t)r * D + d];
            g[i % WGROUPS] = g[i % WGROUPS] + t;
        }
        float s = ((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7]));
        o->Wf[d] = o->Wf[d] + s;
    }
}

/* Detection f(x_s) in the BALANCED kernel's order (apsm_detect.cu:526-538, 690-876):
 * per lane, the linear terms idx = l, l+32, ... first, then Gaussian terms for
 * b = l, l+32, ... ; then the warp shuffle-down tree. */
static float detect_one_f32(const apsm_oracle* o, const float* x)
{
    const apsm_oracle_params* p = &o->par;
    const float ew = -0.5f / p->gaussian_variance;
    float part[LANES];
    memset(part, 0, sizeof(part));
    for (uint32_t idx = 0; idx < o->D; ++idx) {
        float ke = p->linear_weight * x[idx];
        part[idx & (LANES - 1)] = part[idx & (LANES - 1)] + o->Wf[idx] * ke;
    }
    for (uint32_t b = 0; b < o->used; ++b) {
        uint32_t r = phys(o, b);
        const float* d = &o->Xf[(size_t)r * o->D];
        float acc = 0.f;
        for (uint32_t k = 0; k < o->D; ++k) {
            float diff = d[k] - x[k];
            acc = fmaf(diff, diff, acc);
        }
        float ke = o->Af[r] * p->gaussian_weight;
        ke = ke * expf(ew * acc);
        part[b & (LANES - 1)] = part[b & (LANES - 1)] + ke;
    }
    for (uint32_t off = LANES / 2; off >= 1; off >>= 1)
        for (uint32_t l = 0; l < off; ++l) part[l] = part[l] + part[l + off];
    return part[0];
}

/* normConstraint (kernel_adapt_coeffs, apsm_train.cu:190-256, run after every
 * step by :142-145): ||f_G||^2 = sum_i sum_j wG k(d_i, d_j) a_i a_j over the
 * dictionary, summed as the reference does -- block i, lane t over
 * j = t, t+32, ... (((wG k) a_i) a_j, fma-contracted into the lane sum), lanes
 * added in order, then rows in order -- and if its square root exceeds the
 * bound every coefficient is multiplied by bound / norm.  (The reference stages
 * d_j in a 32-float array: dictionary rows wider than 32 features overflow it.) */
static void adapt_coeffs_f32(apsm_oracle* o)
{
    const apsm_oracle_params* p = &o->par;
    const float ew = -0.5f / p->gaussian_variance;
    const uint32_t M = o->used, D = o->D;
    float* rowsum = (float*)malloc((size_t)(M ? M : 1) * sizeof(float));
#pragma omp parallel for schedule(static) if (M > 64)
    for (uint32_t i = 0; i < M; ++i) {
        const uint32_t ri = phys(o, i);
        const float ai = o->Af[ri];
        float lane[LANES];
        memset(lane, 0, sizeof(lane));
        for (uint32_t j = 0; j < M; ++j) {
            const uint32_t rj = phys(o, j);
            const float k = kern_f32(&o->Xf[(size_t)ri * D], &o->Xf[(size_t)rj * D], D, ew);
            const float t = (p->gaussian_weight * k) * ai;
            lane[j % LANES] = fmaf(t, o->Af[rj], lane[j % LANES]);
        }
        float r = 0.f;
        for (uint32_t l = 0; l < LANES && l < M; ++l) r = r + lane[l];
        rowsum[i] = r;
    }
    float norm = 0.f;
    for (uint32_t i = 0; i < M; ++i) norm = norm + rowsum[i];
    free(rowsum);
    if (norm > 0.f) norm = sqrtf(norm);
    if (norm > p->norm_constraint) {
        const float factor = p->norm_constraint / norm;
        for (uint32_t i = 0; i < M; ++i) o->Af[phys(o, i)] *= factor;
    }
}

static void adapt_coeffs_f64(apsm_oracle* o)
{
    const apsm_oracle_params* p = &o->par;
    const double ew = -0.5 / (double)p->gaussian_variance;
    const uint32_t M = o->used, D = o->D;
    double norm = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : norm) if (M > 64)
    for (uint32_t i = 0; i < M; ++i) {
        const uint32_t ri = phys(o, i);
        for (uint32_t j = 0; j < M; ++j) {
            const uint32_t rj = phys(o, j);
            double acc = 0.0;
            for (uint32_t k = 0; k < D; ++k) {
                const double diff = o->Xd[(size_t)ri * D + k] - o->Xd[(size_t)rj * D + k];
                acc += diff * diff;
            }
            norm += (double)p->gaussian_weight * exp(ew * acc) * o->Ad[ri] * o->Ad[rj];
        }
    }
    if (norm > 0.0) norm = sqrt(norm);
    if (norm > (double)p->norm_constraint) {
        const double factor = (double)p->norm_constraint / norm;
        for (uint32_t i = 0; i < M; ++i) o->Ad[phys(o, i)] *= factor;
    }
}

/* computeNormRatio (apsm_noma_detector.cu:220-311): wL |w|^2 / (wG a^T K a), the
 * Gaussian sum as kernel_norm_ratio adds it -- row i by LANES lanes, lane l over
 * j = l, l+LANES, ... ((k a_i) fused with a_j into the lane sum), lanes in order,
 * rows in order -- and the linear sum in order (fma-contracted). */
float apsm_oracle_norm_ratio(const apsm_oracle* o)
{
    const apsm_oracle_params* p = &o->par;
    const float ew = -0.5f / p->gaussian_variance;
    const uint32_t M = o->used, D = o->D;
    float g = 0.f;
    for (uint32_t i = 0; i < M; ++i) {
        const uint32_t ri = phys(o, i);
        float lane[LANES];
        memset(lane, 0, sizeof(lane));
        for (uint32_t j = 0; j < M; ++j) {
            const uint32_t rj = phys(o, j);
            const float k = kern_f32(&o->Xf[(size_t)ri * D], &o->Xf[(size_t)rj * D], D, ew);
            lane[j % LANES] = fmaf(k * o->Af[ri], o->Af[rj], lane[j % LANES]);
        }
        float r = 0.f;
        for (uint32_t l = 0; l < LANES && l < M; ++l) r = r + lane[l];
        g = g + r;
    }
    g = g * p->gaussian_weight;
    float lin = 0.f;
    for (uint32_t d = 0; d < D; ++d) lin = fmaf(o->Wf[d], o->Wf[d], lin);
    lin = lin * p->linear_weight;
    return lin / g;
}

/* ---------------------------------------------------------------- FP64 -- */

static double predict_f64(const apsm_oracle* o, const double* x)
{
    const apsm_oracle_params* p = &o->par;
    const double ew = -0.5 / (double)p->gaussian_variance;
    double lin = 0.0, gau = 0.0;
    for (uint32_t d = 0; d < o->D; ++d) lin += x[d] * o->Wd[d];
    for (uint32_t b = 0; b < o->used; ++b) {
        uint32_t r = phys(o, b);
        const double* dv = &o->Xd[(size_t)r * o->D];
        double acc = 0.0;
        for (uint32_t k = 0; k < o->D; ++k) {
            double diff = dv[k] - x[k];
            acc += diff * diff;
        }
        gau += o->Ad[r] * exp(ew * acc);
    }
    return (double)p->linear_weight * lin + (double)p->gaussian_weight * gau;
}

static void step_f64(apsm_oracle* o, uint32_t start, uint32_t n_active, uint32_t wk, double* f, double* c)
{
    const apsm_oracle_params* p = &o->par;
    const uint32_t D = o->D;
#pragma omp parallel for schedule(static) if (n_active > 8)
    for (uint32_t i = 0; i < n_active; ++i) {
        uint32_t r = phys(o, start + i);
        f[i] = predict_f64(o, &o->Xd[(size_t)r * D]);
    }
    for (uint32_t i = 0; i < n_active; ++i) {
        uint32_t r = phys(o, start + i);
        double e = o->Yd[r] - f[i], cc = 0.0;
        double eB = (double)p->eB;
        if (e > eB) cc = e - eB;
        else if (e < -eB) cc = e + eB;
        double nrm = 0.0;
        for (uint32_t d = 0; d < D; ++d) nrm += o->Xd[(size_t)r * D + d] * o->Xd[(size_t)r * D + d];
        c[i] = cc / (double)wk / ((double)p->linear_weight * nrm + (double)p->gaussian_weight);
    }
    for (uint32_t i = 0; i < n_active; ++i) {
        uint32_t r = phys(o, start + i);
        o->Ad[r] += c[i];
        for (uint32_t d = 0; d < D; ++d) o->Wd[d] += c[i] * o->Xd[(size_t)r * D + d];
    }
}

/* ---------------------------------------------------------------- driver -- */

/* Host step loop of wrapperTrain (apsm_train.cu:100-160).  Rows are staged
 * from the pilots (pushRowsFromMatrix, apsm_train.cu:93) and become visible
 * sampleStep rows per step.  At each step the reference launches
 * min(2q, sample_idx) blocks, the kernel uses window Wk = min(2q, used) and
 * block b updates logical row used - Wk + b (apsm_train.cu:118-119, 333-346).
 * For a call that appends to an existing dictionary the launch count also
 * counts the rows already present, so the window slides on continuously. */
/* Per-step history (NomaTrainHistory, cpp/lib/noma/noma_train_history.cu:65-248;
 * recorded by apsm_train.cu:147-156 after every step): the training rows of this
 * call and the validation samples are detected with the current model and EVM,
 * SER and BER of both are computed in the reference's float order. */
typedef struct {
    const float* rx_val; /* antenna-major complex, S samples */
    const float* tx_val; /* S complex */
    uint32_t S, bps;
    float mod_scale;
    float* out;          /* max_steps x 6: train evm, ser, ber, val evm, ser, ber */
    uint32_t max_steps, n;
} history_ctx;

/* demap1D (noma_train_history.cu:186-196): round half away from zero, clamp, Gray code. */
static uint32_t hist_demap1d(float x, uint32_t num_symbols)
{
    float v = (x + (float)num_symbols - 1.f) / 2.f;
    int32_t xi = (int32_t)roundf(v);
    if (xi < 0) xi = 0;
    if (xi > (int32_t)num_symbols - 1) xi = (int32_t)num_symbols - 1;
    return (uint32_t)(xi ^ (xi >> 1));
}

static int hist_symbol_error_1d(float t, float h, float s, float mx)
{
    return fabsf(t - h) > s && !(h > +mx && t > +mx - s) && !(h < -mx && t < -mx + s);
}

/* kernelComputeEvm / kernelComputeSer(Bpsk) / kernelComputeBer (noma_train_history.cu:96-235):
 * one block of LANES threads, thread l sums symbols l, l+LANES, ... then a halving tree.
 * y_true / y_hat: n symbols, (re, im) interleaved. */
static void hist_metrics(const float* y_true, const float* y_hat, uint32_t n, uint32_t bps, float mod_scale,
                         float* evm, float* ser, float* ber)
{
    float se[LANES], ss[LANES], sb[LANES];
    memset(se, 0, sizeof(se));
    memset(ss, 0, sizeof(ss));
    memset(sb, 0, sizeof(sb));
    const float mx = (float)((1u << (bps / 2)) - 1u) * mod_scale;
    const float rev = (float)(1.0 / (double)mod_scale);
    const uint32_t nsym = bps == 1 ? 2u : 1u << (bps / 2);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t l = i % LANES;
        const float dr = y_true[2 * i] - y_hat[2 * i];
        const float di = y_true[2 * i + 1] - y_hat[2 * i + 1];
        se[l] = se[l] + fmaf(dr, dr, di * di);
        int err;
        if (bps == 1) err = signbit(y_true[2 * i]) != signbit(y_hat[2 * i]);
        else err = hist_symbol_error_1d(y_true[2 * i], y_hat[2 * i], mod_scale, mx) ||
                   hist_symbol_error_1d(y_true[2 * i + 1], y_hat[2 * i + 1], mod_scale, mx);
        ss[l] = ss[l] + (float)err;
        uint32_t b = (uint32_t)__builtin_popcount(hist_demap1d(y_true[2 * i] * rev, nsym) ^
                                                  hist_demap1d(y_hat[2 * i] * rev, nsym));
        sb[l] = sb[l] + (float)b;
        if (bps > 1) {
            b = (uint32_t)__builtin_popcount(hist_demap1d(y_true[2 * i + 1] * rev, nsym) ^
                                             hist_demap1d(y_hat[2 * i + 1] * rev, nsym));
            sb[l] = sb[l] + (float)b;
        }
    }
    for (uint32_t size = LANES / 2; size > 0; size /= 2)
        for (uint32_t l = 0; l < size; ++l) {
            se[l] = se[l] + se[l + size];
            ss[l] = ss[l] + ss[l + size];
            sb[l] = sb[l] + sb[l + size];
        }
    *evm = sqrtf(se[0] / (float)n);
    *ser = ss[0] / (float)n;
    *ber = sb[0] / (float)(n * bps);
}

static void hist_record(apsm_oracle* o, history_ctx* h, const float* staged, const float* ys, uint32_t rows)
{
    if (h->n >= h->max_steps) {
        h->n++;
        return;
    }
    const uint32_t D = o->D;
    const uint32_t nv = 2 * h->S;
    float* est = (float*)malloc((size_t)(rows + nv) * sizeof(float));
    float* yv = (float*)malloc((size_t)nv * sizeof(float));
#pragma omp parallel
    {
        float xf[256];
#pragma omp for schedule(static)
        for (uint32_t r = 0; r < rows + nv; ++r) {
            const float* x = &staged[(size_t)r * D];
            if (r >= rows) {
                dedup_column(h->rx_val, o->n_ant, h->S, r - rows, xf);
                x = xf;
            }
            est[r] = detect_one_f32(o, x);
        }
    }
    for (uint32_t c = 0; c < nv; ++c) yv[c] = h->tx_val[c];
    float* out = &h->out[(size_t)h->n * 6];
    hist_metrics(ys, est, rows / 2, h->bps, h->mod_scale, &out[0], &out[1], &out[2]);
    hist_metrics(yv, est + rows, h->S, h->bps, h->mod_scale, &out[3], &out[4], &out[5]);
    free(est);
    free(yv);
    h->n++;
}

static int train_impl(apsm_oracle* o, const float* rx, const float* tx, uint32_t P, history_ctx* hist);

int apsm_oracle_train(apsm_oracle* o, const float* rx, const float* tx, uint32_t P)
{
    return train_impl(o, rx, tx, P, NULL);
}

int apsm_oracle_train_history(apsm_oracle* o, const float* rx, const float* tx, uint32_t P, const float* rx_val,
                              const float* tx_val, uint32_t S, uint32_t bps, float mod_scale, float* history,
                              uint32_t max_steps, uint32_t* n_steps)
{
    if (!o || o->prec != APSM_ORACLE_F32 || !rx_val || !tx_val || S == 0 || bps == 0 || !history) return 1;
    history_ctx h = {rx_val, tx_val, S, bps, mod_scale, history, max_steps, 0};
    int st = train_impl(o, rx, tx, P, &h);
    if (n_steps) *n_steps = h.n;
    if (st == 0 && h.n > max_steps) return 3;
    return st;
}

static int train_impl(apsm_oracle* o, const float* rx, const float* tx, uint32_t P, history_ctx* hist)
{
    if (!o || !rx || !tx || P == 0) return 1;
    const apsm_oracle_params* p = &o->par;
    const uint32_t D = o->D, rows = 2 * P;
    const uint32_t q2 = 2 * p->window_size, s = p->sample_step;
    if (s == 0 || q2 == 0) return 2;
    float* staged = (float*)malloc((size_t)rows * D * sizeof(float));
    float* ys = (float*)malloc((size_t)rows * sizeof(float));
    for (uint32_t col = 0; col < rows; ++col) {
        dedup_column(rx, o->n_ant, P, col, &staged[(size_t)col * D]);
        ys[col] = tx[col]; /* tx interleaved (re,im) == target of column col */
    }
    uint32_t next = 0;
    const uint32_t m_before = o->used;
    float *ff = NULL, *cf = NULL;
    double *fd = NULL, *cd = NULL;
    if (o->prec == APSM_ORACLE_F32) { ff = (float*)malloc(q2 * sizeof(float)); cf = (float*)malloc(q2 * sizeof(float)); }
    else { fd = (double*)malloc(q2 * sizeof(double)); cd = (double*)malloc(q2 * sizeof(double)); }

    for (uint32_t pass = 0; pass < p->train_passes; ++pass) {
        if (pass == 0 && p->start_full_window) {
            uint32_t k = q2 > s ? q2 - s : 0;
            for (uint32_t i = 0; i < k && next < rows; ++i, ++next) reveal_row(o, &staged[(size_t)next * D], ys[next]);
        }
        for (uint32_t sidx = p->start_full_window ? q2 : s; sidx <= rows; sidx += s) {
            if (pass == 0)
                for (uint32_t i = 0; i < s && next < rows; ++i, ++next) reveal_row(o, &staged[(size_t)next * D], ys[next]);
            uint32_t n_launch = umin(q2, sidx + (pass == 0 ? m_before : 0));
            uint32_t wk = umin(q2, o->used);
            uint32_t start = o->used - wk;
            uint32_t n_active = umin(n_launch, wk);
            if (n_active == 0) continue;
            if (o->prec == APSM_ORACLE_F32) step_f32(o, start, n_active, wk, ff, cf);
            else step_f64(o, start, n_active, wk, fd, cd);
            if (p->norm_constraint > 0.f) {
                if (o->prec == APSM_ORACLE_F32) adapt_coeffs_f32(o);
                else adapt_coeffs_f64(o);
            }
            if (hist) hist_record(o, hist, staged, ys, rows);
        }
    }
    free(ff); free(cf); free(fd); free(cd);
    free(staged);
    free(ys);
    return 0;
}

int apsm_oracle_detect(apsm_oracle* o, const float* rx, uint32_t S, float* est)
{
    if (!o || !rx || !est) return 1;
    const uint32_t D = o->D;
#pragma omp parallel
    {
        float xf[256];
        double xd[256];
#pragma omp for schedule(static)
        for (uint32_t col = 0; col < 2 * S; ++col) {
            dedup_column(rx, o->n_ant, S, col, xf);
            if (o->prec == APSM_ORACLE_F32) {
                est[col] = detect_one_f32(o, xf);
            } else {
                for (uint32_t d = 0; d < D; ++d) xd[d] = (double)xf[d];
                est[col] = (float)predict_f64(o, xd);
            }
        }
    }
    return 0;
}

uint32_t apsm_oracle_rows(const apsm_oracle* o) { return o->used; }

void apsm_oracle_get_state(const apsm_oracle* o, double* dict, double* y, double* a, double* w)
{
    const uint32_t D = o->D;
    for (uint32_t b = 0; b < o->used; ++b) {
        uint32_t r = phys(o, b);
        for (uint32_t d = 0; d < D; ++d)
            if (dict) dict[(size_t)b * D + d] = o->prec == APSM_ORACLE_F32 ? o->Xf[(size_t)r * D + d] : o->Xd[(size_t)r * D + d];
        if (y) y[b] = o->prec == APSM_ORACLE_F32 ? o->Yf[r] : o->Yd[r];
        if (a) a[b] = o->prec == APSM_ORACLE_F32 ? o->Af[r] : o->Ad[r];
    }
    if (w)
        for (uint32_t d = 0; d < D; ++d) w[d] = o->prec == APSM_ORACLE_F32 ? o->Wf[d] : o->Wd[d];
}

int apsm_oracle_set_state(apsm_oracle* o, uint32_t rows, const double* dict, const double* a, const double* w)
{
    if (rows > o->cap) return 1;
    apsm_oracle_reset(o);
    const uint32_t D = o->D;
    for (uint32_t b = 0; b < rows; ++b) {
        for (uint32_t d = 0; d < D; ++d) {
            if (o->prec == APSM_ORACLE_F32) o->Xf[(size_t)b * D + d] = (float)dict[(size_t)b * D + d];
            else o->Xd[(size_t)b * D + d] = dict[(size_t)b * D + d];
        }
        if (o->prec == APSM_ORACLE_F32) o->Af[b] = (float)a[b];
        else o->Ad[b] = a[b];
    }
    for (uint32_t d = 0; d < D; ++d) {
        if (o->prec == APSM_ORACLE_F32) o->Wf[d] = (float)w[d];
        else o->Wd[d] = w[d];
    }
    o->used = rows;
    o->head = 0;
    return 0;
}

void apsm_oracle_set_variance(apsm_oracle* o, float variance) { o->par.gaussian_variance = variance; }

void apsm_oracle_set_w(apsm_oracle* o, const double* w)
{
    for (uint32_t d = 0; d < o->D; ++d) {
        if (o->prec == APSM_ORACLE_F32) o->Wf[d] = (float)w[d];
        else o->Wd[d] = w[d];
    }
}
