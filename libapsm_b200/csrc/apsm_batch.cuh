// Batched (many-detector) APSM kernels: descriptors and declarations.
//
// The batched form works on complex samples ("pairs"): universe pair b is the
// complex received vector y_b (N antennas) behind the reference's two Dedup
// rows 2b = [Re y_b; Im y_b] and 2b+1 = [Im y_b; -Re y_b]
// (cpp/lib/cuda/cuda_matrix_device.cuh:180-188, :288-296).  For two pairs
// b, n with r + i m = y_b^H y_n and squared norms n_b, n_n the four Gaussian
// kernel values of their rows take three distinct values:
//   K(2b, 2n)   = K(2b+1, 2n+1) = wG exp(ew (n_b + n_n - 2 r))   "A"
//   K(2b, 2n+1)                 = wG exp(ew (n_b + n_n - 2 m))   "Bp"
//   K(2b+1, 2n)                 = wG exp(ew (n_b + n_n + 2 m))   "Bm"
// and the linear kernel <x_2b, x_2n> = <x_2b+1, x_2n+1> = r,
// <x_2b, x_2n+1> = m, <x_2b+1, x_2n> = -m.
#pragma once

#include "apsm_common.cuh"

namespace apsm {

// Settings shared by every job of a batch (one algorithm config).
struct BatchCommon {
    float wL, wG, eB;
    int qP;   // window length in pairs (windowSize)
    int sp;   // pairs entering per step (sampleStep / 2)
    int LB;   // pairs of a column that enter the window kernel: qP + sp
    int XSP;  // pair slots of the sweep's window ring: qP + 3 sp
    int XSPp; // pitch (floats) of the window kernel planes, multiple of 4, >= XSP
    int Np;   // largest complex row pitch of the jobs (float2 units)
};

// One training job: a detector's universe (dictionary pairs already present,
// then the new pilots) swept by one CTA.
struct BatchTrainJob {
    const float2* Y;     // nP x Np universe samples (pair b = complex y_b)
    const float* nrm;    // nP squared norms
    const float* y;      // 2 nP targets (row form: Re x, Im x)
    float* a;            // 2 nP coefficients (row form); in: old rows, out: visible rows
    float* w;            // 2N linear weights (in/out)
    float* r;            // 2N residual weights r = w - sum_{b visible} a_b x_b (in/out, kept with the detector)
    const float4* Kc;    // combined kernel columns (A + wL r, Bp + wL m, Bm - wL m, 0), pairs n in [n_first, nP)
    const TrainStep* steps;
    int n_steps;
    int nP, N, Np, capP; // universe pairs, antennas, row pitch (float2), dictionary capacity in pairs
    int n_first;         // first pair with a kernel column
    int used_beforeP;    // pairs present before this call
    long long kc_base;   // column_prefix(n_first)
    float ew;            // -0.5 / (variance * N^2)
    int fresh;           // start from a fresh state (w = 0; the universe holds only the new pilots)
    // Sums over the old pairs of a call that appends (null otherwise), for every kernel column
    // n in [n_first, nP), per pass of kKcolRows column entries ([n - n_first][pass], pro_stride
    // passes), written by launch_batch_kcol: sum_b a_b Kt(b, n) over b in [pro_lo, pro_hi) for
    // the first window's pairs n < n_first + pro_w (their starting predictions), over
    // b in [col_begin(n), n_first) for the later pairs (the part of their frozen sums whose
    // coefficients this call never changes).
    float2* pro;
    int pro_w, pro_lo, pro_hi, pro_stride;
};

// Kernel-column launch shape: columns per block and column entries per pass.
constexpr int kKcolGroup = 8;
constexpr int kKcolRows = 128;

// Column n holds pairs [col_begin(n), col_end(n)).
__host__ __device__ inline int col_begin(int n, int capP) { return n + 1 - capP > 0 ? n + 1 - capP : 0; }
__host__ __device__ inline int col_end(int n, int qP, int nP) { return n + qP < nP ? n + qP : nP; }

// Range of old pairs summed into the pro sums of column n.
__host__ __device__ inline void pro_range(const BatchTrainJob& j, int n, int* lo, int* hi)
{
    if (n < j.n_first + j.pro_w) {
        *lo = j.pro_lo;
        *hi = j.pro_hi;
    } else {
        *lo = col_begin(n, j.capP);
        *hi = j.n_first;
    }
}

// Sum of the column lengths of pairs [0, n) (closed form of the clamped ramps).
__host__ __device__ inline long long column_prefix(long long n, long long qP, long long nP, long long capP)
{
    long long k = nP - qP;
    if (k < 0) k = 0;
    if (k > n) k = n;
    const long long s1 = k * qP + k * (k - 1) / 2 + (n - k) * nP;
    const long long j = n - capP > 0 ? n - capP : 0;
    return s1 - j * (j + 1) / 2;
}

// One detection job: S data samples of one detector against its dictionary.
struct BatchDetectJob {
    const float2* rx;   // N x S received data samples, antenna-major (as the caller holds them)
    const float2* Yd;   // Mp x Np dictionary samples
    const float* nrm_d; // Mp norms
    const float* a;     // 2 Mp coefficients (row form)
    const float* w;     // 2N linear weights
    float2* out;        // S soft estimates (Re = f(row 2s), Im = f(row 2s+1))
    int S, Mp, N, Np;
    float ew;
    // split launches (parts > 1): per-chunk partial sums [chunk][S] and one
    // arrival counter per sample tile (zeroed before the launch)
    float2* part;
    int* cnt;
};

// One detection job on the tensor cores (kernels_batch_gram.cu).
struct BatchGramJob {
    const float2* rx;   // N x S data samples, antenna-major (as the caller holds them)
    float* nrm_s;       // S squared norms (written by the operand packing)
    const float* w;     // 2N linear weights
    float2* lin;        // S: wL <w, x_2s>, wL <w, x_2s+1>
    uint8_t* a_ops;     // ceil(S / 128) sample tiles, UMMA canonical layout (hi [| lo] of the Gram form)
    const float2* Yd;   // Mp x Np dictionary samples
    const float* nrm_d; // Mp norms
    const float* a;     // 2 Mp coefficients
    uint8_t* b_ops;     // n_chunks dictionary chunks (64 pairs = 128 rows), same layout
    float* bx;          // n_chunks x (128 a*wG + 64 norms)
    float2* out;        // S soft estimates
    int S, N, Np, Kp, Mp, n_chunks;
    float ew2;          // ew * log2(e)
};

// One training job of a tensor-core kernel-column launch (kernels_batch_kcol_tc.cu): its
// universe pairs as UMMA operands (TF32 hi | lo, canonical K-major): row tiles of 128 pairs
// b in [0, nP) and column chunks of 64 pairs n in [n_first, nP) (two rows per pair).
struct BatchKcolTcJob {
    const float2* Y;    // nP x Np universe pairs
    const float* nrm;   // nP pair norms
    float4* Kc;         // the job's kernel columns (as BatchTrainJob::Kc)
    uint8_t* a_ops;     // a_tiles row tiles
    uint8_t* b_ops;     // b_chunks column chunks
    float* a_nrm;       // a_tiles x 128 row norms (0 past nP)
    int nP, N, Np, Kp, capP, n_first, a_tiles, b_chunks;
    long long kc_base;  // column_prefix(n_first)
    float ewl2;         // ew log2(e)
};

// Packing of complex samples: antenna-major rx (N x L complex) -> L x Np pairs + norms.
struct BatchPackJob {
    const float2* rx;   // N x L
    const float2* tx;   // L targets or null
    const int* perm;    // sample order or null
    float2* Y;          // destination pairs
    float* nrm;         // destination norms
    float* y;           // destination targets (2 per sample) or null
    float* a;           // coefficients to zero (2 per sample) or null
    int L, N, Np;
};

// Copy of a detector's resident dictionary into (or out of) a universe.
struct BatchCopyJob {
    const float2* Ysrc; const float* nsrc; const float* ysrc; const float* asrc;
    float2* Ydst; float* ndst; float* ydst; float* adst;
    int pairs, Np;
};

// A pool detector's state (pairs Y (pitch Np), row-form targets and coefficients, `rows` =
// 2 x pairs) as the single detector's Dedup rows (pitch Dp, with their squared norms), and
// back: the pool runs training jobs of normConstraint configs with the single detector's
// exact sweep.
cudaError_t launch_pool_to_rows(const float2* Y, int Np, const float* y, const float* a, int rows, int N, int Dp,
                                float* X, float* nrm, float* dy, float* da, cudaStream_t s);
cudaError_t launch_rows_to_pool(const float* X, const float* nrm, const float* dy, const float* da, int rows, int N,
                                int Dp, int Np, float2* Y, float* pn, float* y, float* a, cudaStream_t s);

// max_n: largest antenna count of the jobs (sizes the kernel's shared memory)
// max_blocks > 0 bounds the grid (blocks then loop over the (job, chunk) units)
cudaError_t launch_batch_pack(const BatchPackJob* d_jobs, int n_jobs, int max_len, int max_n, cudaStream_t s,
                              int max_blocks = 0);
cudaError_t launch_batch_copy(const BatchCopyJob* d_jobs, int n_jobs, int max_pairs, int max_np, cudaStream_t s);
// row_split: blocks per column group, each taking every row_split-th pass of
// kColRows column entries (entries are computed alike whatever the split).
// order (device, n_jobs entries, or null for 0..n_jobs-1): the jobs of the
// launch as indices into d_jobs; the pool launches one antenna class at a
// time, so each launch's kernel keeps rows of its class's size in registers.
cudaError_t launch_batch_kcol(const BatchTrainJob* d_jobs, const int* order, int n_jobs, int max_cols, int max_n,
                              int row_split, BatchCommon cm, cudaStream_t s);
int batch_kcol_group(); // columns per block
int batch_kcol_rows();  // column entries per block pass
// The same columns with the cross terms y_b^H y_n on the tensor cores (TF32 split, FP32
// accuracy), for jobs without old-pair sums (pro == null) and N <= 32: operand packing, then
// one CTA per chunk of 64 columns (chunk_prefix[j] = first CTA of job j), Kpmax the largest Kp
// of the launch.
int batch_kcol_tc_kp(int N);
int batch_kcol_tc_row_tile();  // pairs per row tile
int batch_kcol_tc_col_pairs(); // columns per chunk (CTA)
size_t batch_kcol_tc_a_bytes(int Kp);
size_t batch_kcol_tc_b_bytes(int Kp);
cudaError_t launch_batch_kcol_tc(const BatchKcolTcJob* d_jobs, int n_jobs, int max_units, const int* d_chunk_prefix,
                                 int total_chunks, int Kpmax, BatchCommon cm, int* d_err, cudaStream_t s);
size_t batch_sweep_smem(const BatchCommon& cm);
int batch_sweep_threads();
cudaError_t batch_sweep_occupancy(const BatchCommon& cm, int* ctas_per_sm);
cudaError_t launch_batch_sweep(const BatchTrainJob* d_jobs, int n_jobs, BatchCommon cm, int grid, int* d_counter,
                               int* d_err, cudaStream_t s);
// Jobs of one antenna class (N <= nmax, nmax in {4, 8, 16, 32, 64}).
// parts: blocks that share one tile of samples, each taking a contiguous run of
// the job's 64-pair dictionary chunks (1: one block per tile).  Results do not
// depend on parts: every chunk's sum starts from zero and the chunk sums are
// added in chunk order, by the block itself or by the tile's last block.
cudaError_t launch_batch_detect(const BatchDetectJob* d_jobs, int n_jobs, int max_tiles, int parts, int nmax, float wL,
                                float wG, cudaStream_t s);
int batch_detect_tile();  // samples per block of launch_batch_detect
int batch_detect_chunk(); // dictionary pairs per chunk of launch_batch_detect

// Tensor-core detection of jobs with Kp <= Kp_max in one Gram form `mode`
// (GramMode: kBF16, kBF16x3, kTF32, kTF32x3).  Kp = 2N rounded up to the K of
// one UMMA (8 TF32 or 16 BF16 elements), Kp_max in {8, 16, 32, 64}: operand
// packing and the Gram kernel, whose CTA t works on tile t - tile_prefix[j]
// of job j.
int batch_gram_tile();        // samples per tile
int batch_gram_chunk_pairs(int mode, int Kp); // dictionary pairs per chunk (64, or 32 for TF32 hi/lo above 32 features)
int batch_gram_kp(int mode, int N);
size_t batch_gram_a_bytes(int mode, int Kp);
size_t batch_gram_b_bytes(int mode, int Kp);
size_t batch_gram_bx_floats(int mode, int Kp);
// stages: dictionary chunks in flight, 2 or 3 (0: the built-in choice; 3 only where it fits)
cudaError_t launch_batch_gram(int mode, const BatchGramJob* d_jobs, int n_jobs, int max_tiles, int max_chunks,
                              const int* d_tile_prefix, int total_tiles, int Kp_max, float wL, float wG, int* d_err,
                              int stages, cudaStream_t s);

} // namespace apsm
