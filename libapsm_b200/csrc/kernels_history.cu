// Training history on B200: the reference's NomaTrainHistory
// (cpp/lib/noma/noma_train_history.cu:65-248), filled by the training loop
// after every step (cpp/lib/apsm/apsm_train.cu:147-156): the model of that
// step detects the call's training rows and a validation set, and EVM, SER
// and BER of both are recorded.
//
// The reference runs, per step, two detections and six single-block metric
// kernels, each followed by a host synchronisation.  Here the sweep only
// stores each step's model (the coefficients of the rows it updated and the
// linear weights, TrainArgs::snap_a / snap_w) and three kernels evaluate every
// step at once afterwards:
//   history_expand_kernel  per-step coefficients -> dense A[step][row] over the
//                          universe rows (0 where a row is not in that step's
//                          dictionary);
//   history_eval_kernel    est[step][j] = sum_b A[step][b] wG k(x_b, e_j)
//                          + wL <w_step, e_j> for 64 steps x 64 evaluation rows
//                          per block (kernel values computed once per block and
//                          shared by its 64 steps; dictionary chunks outside
//                          the block's steps' dictionaries are skipped), with
//                          the metric partial sums of each symbol pair reduced
//                          in the block -- estimates never reach memory;
//   history_reduce_kernel  partial sums of the tiles in a fixed order, then
//                          EVM = sqrt(sum |e|^2 / n), SER = errors / n,
//                          BER = bit errors / (n bps).
// Metrics follow the reference kernels: SER from symbolError1D on both axes
// (BPSK: sign of the real part), BER from demap1D of est * (1 / scale) and the
// popcount of the Gray-code difference.
#include "apsm_kernels.cuh"

namespace apsm {

namespace {

constexpr int kRows = 64;   // evaluation rows per block (32 symbols)
constexpr int kSteps = 64;  // steps per block
constexpr int kChunk = 32;  // dictionary rows per chunk
constexpr int kThreads = 256;

__device__ __forceinline__ uint32_t demap_1d(float x, uint32_t num_symbols)
{
    // demap1D (noma_train_history.cu:186-196)
    int xi = int(roundf((x + float(num_symbols) - 1.f) / 2.f));
    xi = min(int(num_symbols) - 1, max(0, xi));
    return uint32_t(xi ^ (xi >> 1));
}

__device__ __forceinline__ bool symbol_error_1d(float t, float h, float s, float mx)
{
    // symbolError1D (noma_train_history.cu:130-136)
    return fabsf(t - h) > s && !(h > +mx && t > +mx - s) && !(h < -mx && t < -mx + s);
}

} // namespace

__global__ void history_expand_kernel(HistoryArgs h)
{
    const int u = blockIdx.y;
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= h.nU) return;
    float cur = b < h.used_before ? h.a0[size_t(u) * h.a0_stride + b] : 0.f;
    const float* sa = h.snap_a + size_t(u) * h.n_steps * h.q2;
    float* A = h.A + size_t(u) * h.n_steps * h.nU;
    for (int t = 0; t < h.n_steps; ++t) {
        const TrainStep st = h.steps[t];
        const int start = st.hi - st.wk;
        if (b >= start && b < start + st.n_active) cur = sa[size_t(t) * h.q2 + (b - start)];
        else if (h.snap_scale) cur *= h.snap_scale[size_t(u) * h.n_steps + t]; // normConstraint of step t
        const int lo = max(0, st.hi - h.cap);
        A[size_t(t) * h.nU + b] = (b >= lo && b < st.hi) ? cur : 0.f;
    }
}

// Shared memory (floats): es[kRows][EP] evaluation rows, xs[kChunk][EP] dictionary
// rows, kc[kChunk][kRows] kernel values, as[kSteps][kChunk + 1] coefficients,
// EP = D + 1 (odd pitch: the per-row difference loops are conflict-free).
__global__ void __launch_bounds__(kThreads) history_eval_kernel(HistoryArgs h)
{
    const int tile = blockIdx.x, t0 = blockIdx.y * kSteps, u = blockIdx.z;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int D = h.D, EP = D + 1;
    extern __shared__ __align__(16) float smem[];
    float* es = smem;
    float* xs = es + kRows * EP;
    float* kc = xs + kChunk * EP;
    float* as = kc + kChunk * kRows;
    __shared__ int s_lo, s_hi;

    const int r0 = tile * kRows;
    for (int i = tid; i < kRows * D; i += kThreads) {
        const int r = i / D, d = i - r * D;
        es[r * EP + d] = r0 + r < h.nE ? h.E[size_t(r0 + r) * h.Dp + d] : 0.f;
    }
    if (tid == 0) {
        int lo = h.nU, hi = 0;
        for (int t = t0; t < min(h.n_steps, t0 + kSteps); ++t) {
            const TrainStep st = h.steps[t];
            lo = min(lo, max(0, st.hi - h.cap));
            hi = max(hi, st.hi);
        }
        s_lo = lo;
        s_hi = hi;
    }
    __syncthreads();

    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[i][k] = 0.f;

    const float* A = h.A + size_t(u) * h.n_steps * h.nU;
    const ModelParams mp = h.mp;
    for (int b0 = s_lo / kChunk * kChunk; b0 < s_hi; b0 += kChunk) {
        for (int i = tid; i < kChunk * D; i += kThreads) {
            const int r = i / D, d = i - r * D;
            xs[r * EP + d] = b0 + r < h.nU ? h.X[size_t(b0 + r) * h.Dp + d] : 0.f;
        }
        for (int i = tid; i < kSteps * kChunk; i += kThreads) {
            const int ti = i / kChunk, bi = i - ti * kChunk;
            const int t = t0 + ti, b = b0 + bi;
            as[ti * (kChunk + 1) + bi] = (t < h.n_steps && b < h.nU) ? A[size_t(t) * h.nU + b] : 0.f;
        }
        __syncthreads();
        // kernel values: a warp takes one dictionary row against 32 evaluation rows
        for (int i = tid; i < kChunk * kRows; i += kThreads) {
            const int bi = i / kRows, j = i - bi * kRows;
            const float* xb = xs + bi * EP;
            const float* ej = es + j * EP;
            float dist = 0.f;
            for (int d = 0; d < D; ++d) {
                const float diff = xb[d] - ej[d];
                dist = fmaf(diff, diff, dist);
            }
            kc[bi * kRows + j] = mp.wG * expf(mp.ew * dist);
        }
        __syncthreads();
#pragma unroll 4
        for (int bi = 0; bi < kChunk; ++bi) {
            const float4 kv = *reinterpret_cast<const float4*>(kc + bi * kRows + 4 * tx);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float a = as[(4 * ty + i) * (kChunk + 1) + bi];
                acc[i][0] = fmaf(a, kv.x, acc[i][0]);
                acc[i][1] = fmaf(a, kv.y, acc[i][1]);
                acc[i][2] = fmaf(a, kv.z, acc[i][2]);
                acc[i][3] = fmaf(a, kv.w, acc[i][3]);
            }
        }
        __syncthreads();
    }

    // linear part wL <w_t, e_j>, then the metrics of this thread's two symbols
    const float s = h.mod_scale, mx = h.max_val, rev = h.rev_scale;
    const uint32_t nsym = h.bps == 1 ? 2u : 1u << (h.bps / 2);
    const float* Ey = h.Ey + size_t(u) * h.nE;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int t = t0 + 4 * ty + i;
        float m[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (t < h.n_steps) {
            const float* w = h.snap_w + (size_t(u) * h.n_steps + t) * D;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                float lin = 0.f;
                const float* ej = es + (4 * tx + k) * EP;
                for (int d = 0; d < D; ++d) lin = fmaf(__ldg(w + d), ej[d], lin);
                acc[i][k] = fmaf(mp.wL, lin, acc[i][k]);
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int r = r0 + 4 * tx + 2 * q;
                if (r >= h.nE) continue;
                const float tr = Ey[r], ti = Ey[r + 1];
                const float er = acc[i][2 * q], ei = acc[i][2 * q + 1];
                const float dr = tr - er, di = ti - ei;
                const float e2 = fmaf(dr, dr, di * di);
                bool err;
                if (h.bps == 1) err = signbit(tr) != signbit(er);
                else err = symbol_error_1d(tr, er, s, mx) || symbol_error_1d(ti, ei, s, mx);
                float bits = float(__popc(demap_1d(tr * rev, nsym) ^ demap_1d(er * rev, nsym)));
                if (h.bps > 1) bits += float(__popc(demap_1d(ti * rev, nsym) ^ demap_1d(ei * rev, nsym)));
                if (r < h.n_train) {
                    m[0] += e2;
                    m[1] += err ? 1.f : 0.f;
                    m[2] += bits;
                } else {
                    m[3] += e2;
                    m[4] += err ? 1.f : 0.f;
                    m[5] += bits;
                }
            }
        }
        // sum over the 16 threads of this step row (one half-warp)
#pragma unroll
        for (int c = 0; c < 6; ++c)
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) m[c] += __shfl_xor_sync(0xffffffffu, m[c], o);
        if (tx == 0 && t < h.n_steps) {
            float* out = h.part + ((size_t(u) * h.n_steps + t) * h.n_tiles + tile) * 6;
#pragma unroll
            for (int c = 0; c < 6; ++c) out[c] = m[c];
        }
    }
}

__global__ void history_reduce_kernel(HistoryArgs h)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x; // u * n_steps + t
    if (idx >= h.users * h.n_steps) return;
    const float* p = h.part + size_t(idx) * h.n_tiles * 6;
    float m[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int k = 0; k < h.n_tiles; ++k)
#pragma unroll
        for (int c = 0; c < 6; ++c) m[c] += p[k * 6 + c];
    const float nt = float(h.n_train / 2), nv = float((h.nE - h.n_train) / 2);
    float* out = h.out + size_t(idx) * 6;
    out[0] = sqrtf(m[0] / nt);
    out[1] = m[1] / nt;
    out[2] = m[2] / float((h.n_train / 2) * h.bps);
    out[3] = sqrtf(m[3] / nv);
    out[4] = m[4] / nv;
    out[5] = m[5] / float(((h.nE - h.n_train) / 2) * h.bps);
}

size_t history_eval_smem(int D)
{
    return sizeof(float) * (size_t(kRows + kChunk) * (D + 1) + size_t(kChunk) * kRows + size_t(kSteps) * (kChunk + 1));
}

int history_tiles(int nE) { return (nE + kRows - 1) / kRows; }

cudaError_t launch_history(const HistoryArgs& h, cudaStream_t s)
{
    if (h.n_steps == 0) return cudaSuccess;
    history_expand_kernel<<<dim3((h.nU + 255) / 256, h.users), 256, 0, s>>>(h);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t smem = history_eval_smem(h.D);
    e = cudaFuncSetAttribute(history_eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    history_eval_kernel<<<dim3(h.n_tiles, (h.n_steps + kSteps - 1) / kSteps, h.users), kThreads, smem, s>>>(h);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int n = h.users * h.n_steps;
    history_reduce_kernel<<<(n + 255) / 256, 256, 0, s>>>(h);
    return cudaGetLastError();
}

} // namespace apsm
