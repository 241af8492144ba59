// Tensor-core Gram detection on B200 (tcgen05 / TMEM / bulk async copies).
//
// The detection model (cpp/lib/apsm/apsm_detect.cu:690-876)
//   f_u(x_s) = wL <w_u, x_s> + sum_b (a_ub wG) exp(ew ||d_b - x_s||^2)
// is recast with ||d - x||^2 = ||x||^2 + ||d||^2 - 2 x.d: the cross terms of a
// 128-sample tile against a 256-row dictionary chunk are one UMMA
// (tcgen05.mma, M=128, N=256, FP32 accumulators in tensor memory), the norms
// stay FP32, and the epilogue warps read the accumulator tile (tcgen05.ld),
// form the squared distance, exponentiate on the SFU (ex2.approx) and
// contract with every user's coefficients.  Operand precision:
//   gram_bf16    x.d from BF16 operands (1 product)
//   gram_bf16x3  compensated: x = xh + xl, d = dh + dl (BF16 each);
//                x.d ~ xh.dh + xh.dl + xl.dh (3 products, ~2^-16 relative)
//   gram_tf32    TF32 operands (1 product)
//   gram_tf32x3  compensated TF32 split (3 products, ~FP32 accuracy)
// The squared distance is clamped at 0.  Compensated cross terms (the
// single-product forms bf16 / tf32): rounding both operands to the format's
// unit u moves x.d by at most 2u |x||d|, the base-2 exponent
// ew log2(e) (|x|^2 + |d|^2 - 2 x.d) by at most 2u |es| (es = ew log2(e)
// (|x|^2 + |d|^2)), and a kernel value's contribution to user u's output by at
// most |a_u wG| k ln2 2u |es|.  Where cancellation bites (near-duplicate
// points: x.d ~ (|x|^2 + |d|^2) / 2 with k near 1) the epilogue flags the
// entries whose bound, with the largest coefficient of the row over the
// users, exceeds kFixEps, and recomputes their squared distance exactly as
// sum (x - d)^2 in FP32 from the rows themselves.  Each CTA owns one tile of
// data rows and a contiguous range of dictionary chunks; partial sums per
// range are combined in a fixed order by gram_finish_kernel, so results are
// deterministic.
//
// Roles (320 threads): warps 0-7 epilogue (warp w reads TMEM lanes
// 32*(w%4).., columns of half w/4 of each chunk), warp 8 producer (bulk copies
// of dictionary chunks into a 3-stage ring), warp 9 TMEM allocator and MMA
// issuer.  Every mbarrier wait is bounded; on expiry the kernel records an
// error, stops issuing work, still releases its tensor memory and returns.
#include "apsm_gram.cuh"
#include "apsm_kernels.cuh"
#include "apsm_tc.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>
#include <string>

namespace apsm {

constexpr int kTileM = 128;       // data rows per CTA tile (UMMA M)
constexpr int kMaxStages = 3;     // dictionary chunk ring (2 where 3 stages do not fit)
constexpr int kEpiWarps = 8;
constexpr int kThreads = (kEpiWarps + 2) * 32;
constexpr int kMaxUsers = 16;

struct GramWorkspace {
    DevBuf<uint8_t> a_ops, b_ops, w_ops; // operand tiles in the UMMA canonical K-major layout
    DevBuf<float> xn, dn, aw, part, fw, gate;
    DevBuf<int> err;
    int* h_err = nullptr;
};

void gram_workspace_free(GramWorkspace* g)
{
    if (!g) return;
    if (g->h_err) cudaFreeHost(g->h_err);
    delete g;
}

namespace {

using namespace tc;

// ------------------------------------------------------ operand packing --

// rows: n x Dp fp32.  Writes tiles of R rows: element (r, k) of tile t at byte
// t*R*KE*elem + (k/kc)*(R*16) + (r/8)*128 + (r%8)*16 + (k%kc)*elem, where the
// K extent KE = Kp (hi part) [+ Kp (lo part) for split modes]; rows >= n and
// features >= D are zero.  Also the FP32 squared norms.
template <int MODE>
__global__ void gram_pack_kernel(const float* __restrict__ rows, int n, int Dp, int D, int Kp, int R, int n_tiles,
                                 uint8_t* __restrict__ ops, float* __restrict__ norms)
{
    using T = OpTraits<MODE>;
    const int KE = T::kSplit ? 2 * Kp : Kp;
    const size_t total = size_t(n_tiles) * R * Kp;
    for (size_t idx = blockIdx.x * size_t(blockDim.x) + threadIdx.x; idx < total; idx += size_t(gridDim.x) * blockDim.x) {
        const int k = int(idx % Kp);
        const size_t rr = idx / Kp;
        const int r = int(rr % R), t = int(rr / R);
        const int row = t * R + r;
        const float x = (row < n && k < D) ? rows[size_t(row) * Dp + k] : 0.f;
        float hi, lo;
        split_operand<MODE>(x, &hi, &lo);
        uint8_t* tile = ops + size_t(t) * R * KE * T::kElem;
        put_operand<MODE>(tile, R, r, k, hi);
        if constexpr (T::kSplit) put_operand<MODE>(tile, R, r, Kp + k, lo);
    }
    if (norms) {
        for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
            float acc = 0.f;
            for (int k = 0; k < D; ++k) {
                const float v = rows[size_t(row) * Dp + k];
                acc = fmaf(v, v, acc);
            }
            norms[row] = acc;
        }
    }
}

// per-entry error a flagged entry would exceed (soft-output units) in the single-product forms
constexpr float kFixEps = 1.0f / 8192.0f;

// ln 2 * 2u / kFixEps of a mode's operand rounding unit u (0: split forms, no correction)
template <int MODE> __host__ __device__ constexpr float fix_scale()
{
    return MODE == kBF16 ? 0.69314718f * (2.0f / 256.0f) / kFixEps
                         : (MODE == kTF32 ? 0.69314718f * (2.0f / 2048.0f) / kFixEps : 0.0f);
}

// Fix weights of the compensated forms: fw[b] = max_u |a_u[b] wG| ln2 2u / kFixEps (0 past M)
// and per chunk of N dictionary rows gate[c] = (max fw, max fw |ewl2 dn[b]|, 0, 0).
template <int MODE>
__global__ void __launch_bounds__(256) gram_fix_kernel(const float* __restrict__ a, size_t a_stride, int users, int M,
                                                       int N, float wG, float ewl2, const float* __restrict__ dn,
                                                       float* __restrict__ fw, float* __restrict__ gate)
{
    __shared__ float red[2][8];
    const int c = blockIdx.x;
    float g0 = 0.f, g1 = 0.f;
    for (int k = threadIdx.x; k < N; k += blockDim.x) {
        const int b = c * N + k;
        float v = 0.f;
        if (b < M) {
            for (int u = 0; u < users; ++u) v = fmaxf(v, fabsf(__fmul_rn(a[size_t(u) * a_stride + b], wG)));
            v *= fix_scale<MODE>();
        }
        fw[b] = v;
        g0 = fmaxf(g0, v);
        g1 = fmaxf(g1, v * fabsf(ewl2 * dn[b]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        g0 = fmaxf(g0, __shfl_xor_sync(0xffffffffu, g0, o));
        g1 = fmaxf(g1, __shfl_xor_sync(0xffffffffu, g1, o));
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = g0;
        red[1][threadIdx.x >> 5] = g1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < int(blockDim.x >> 5); ++w) {
            g0 = fmaxf(g0, red[0][w]);
            g1 = fmaxf(g1, red[1][w]);
        }
        gate[4 * c] = g0;
        gate[4 * c + 1] = g1;
        gate[4 * c + 2] = 0.f;
        gate[4 * c + 3] = 0.f;
    }
}

// Exact squared distance of two FP32 rows (16-byte aligned, D features), in feature order.
__device__ __forceinline__ float row_distance(const float* __restrict__ x, const float* __restrict__ d, int D)
{
    float acc = 0.f;
    int k = 0;
    for (; k + 4 <= D; k += 4) {
        const float4 xv = *reinterpret_cast<const float4*>(x + k);
        const float4 dv = *reinterpret_cast<const float4*>(d + k);
        acc = fmaf(xv.x - dv.x, xv.x - dv.x, acc);
        acc = fmaf(xv.y - dv.y, xv.y - dv.y, acc);
        acc = fmaf(xv.z - dv.z, xv.z - dv.z, acc);
        acc = fmaf(xv.w - dv.w, xv.w - dv.w, acc);
    }
    for (; k < D; ++k) acc = fmaf(x[k] - d[k], x[k] - d[k], acc);
    return acc;
}

// aw[u][b] = a_u[b] * wG (the reference's coeff * gaussianKernelWeight), 0 past M.
__global__ void gram_coeff_kernel(const float* __restrict__ a, size_t a_stride, int users, int M, int Mpad, float wG,
                                  float* __restrict__ aw)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= users * Mpad) return;
    const int u = i / Mpad, b = i % Mpad;
    aw[i] = b < M ? __fmul_rn(a[size_t(u) * a_stride + b], wG) : 0.f;
}

struct GramArgs {
    const uint8_t* a_ops; // data tiles (kTileM rows)
    const uint8_t* b_ops; // dictionary chunks (N rows)
    const float* xn;      // data norms
    const float* dn;      // dictionary norms (Mpad)
    const float* aw;      // users x Mpad
    const float* fw;      // fix weights (Mpad)
    const float* gate;    // per chunk: max fw, max fw |ewl2 dn|, 0, 0
    const float* xrows;   // data rows (n_samples x Dp, FP32) for the exact recompute
    const float* drows;   // dictionary rows (M x Dp, FP32)
    float* part;          // splits x users x n_samples partial sums
    int* err;
    int n_samples, Mpad, users, Kp, N, Dp, D;
    int chunks_per_split, n_chunks;
    int stages; // dictionary chunks in flight (<= kMaxStages)
    float ewl2; // ew * log2(e)
    unsigned long long wait_ns; // limit of the bounded waits
};

// NC accumulator columns of one data row: squared distance from the cross term
// and the norms, Gaussian value, contraction with every user's coefficients.
// xs: the stage's norms (xs[0 .. NC)), coefficient rows (xs[(1 + u) N + ...]) and
// fix weights (xs[(1 + users) N + ...]).  CHECK: entries whose error bound exceeds
// kFixEps are left out and returned as bits of the mask (column j -> bit j).
template <int NC, int NU, bool CHECK>
__device__ __forceinline__ uint32_t epilogue_columns(const float* gv, const float* xs, int N, float xn, float ewl2,
                                                     int users, float* acc)
{
    uint32_t mask = 0u;
#pragma unroll
    for (int j = 0; j < NC; j += 4) {
        const float4 dn4 = *reinterpret_cast<const float4*>(xs + j);
        const float t[4] = {xn + dn4.x, xn + dn4.y, xn + dn4.z, xn + dn4.w};
        float kv[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) kv[e] = ex2(ewl2 * fmaxf(fmaf(-2.f, gv[j + e], t[e]), 0.f));
        if constexpr (CHECK) {
            const float4 fw4 = *reinterpret_cast<const float4*>(xs + (1 + users) * N + j);
            const float fw[4] = {fw4.x, fw4.y, fw4.z, fw4.w};
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (kv[e] * (ewl2 * t[e]) * fw[e] < -1.f) {
                    mask |= 1u << (j + e);
                    kv[e] = 0.f;
                }
        }
#pragma unroll
        for (int u = 0; u < NU; ++u) {
            if (u < users) {
                const float4 a4 = *reinterpret_cast<const float4*>(xs + (1 + u) * N + j);
                acc[u] = fmaf(a4.x, kv[0], acc[u]);
                acc[u] = fmaf(a4.y, kv[1], acc[u]);
                acc[u] = fmaf(a4.z, kv[2], acc[u]);
                acc[u] = fmaf(a4.w, kv[3], acc[u]);
            }
        }
    }
    return mask;
}

// Largest |ewl2 xn| of the warp's rows.
__device__ __forceinline__ float warp_exn_max(float ewl2, float xn)
{
    float v = fabsf(ewl2 * xn);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <int MODE, int NU>
__global__ void __launch_bounds__(kThreads, 1) gram_detect_kernel(GramArgs g)
{
    using T = OpTraits<MODE>;
    extern __shared__ __align__(1024) uint8_t smem[];
    const int KE = T::kSplit ? 2 * g.Kp : g.Kp;
    const uint32_t a_bytes = uint32_t(kTileM) * KE * T::kElem;
    const uint32_t b_bytes = uint32_t(g.N) * KE * T::kElem;
    const uint32_t x_bytes = uint32_t(g.N) * 4 * (2 + g.users) + 16; // dn, aw rows, fw, chunk gate
    uint8_t* sA = smem;
    uint8_t* sB = sA + a_bytes;
    const int NS = g.stages;
    float* sX = reinterpret_cast<float*>(sB + size_t(NS) * b_bytes); // [stage][1 + users][N]
    uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(sX) + size_t(NS) * x_bytes);
    uint64_t* full = bars;            // [NS]
    uint64_t* empty = bars + NS;      // [NS]
    uint64_t* tfull = bars + 2 * NS;  // [2]
    uint64_t* tempty = tfull + 2;          // [2]
    uint64_t* afull = tempty + 2;          // [1]
    uint64_t* done = afull + 1;            // [1] all MMAs of the CTA completed
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    float* red = reinterpret_cast<float*>(tmem_slot + 4); // [4 warps][32][users] second-half partials

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x, split = blockIdx.y;
    const int c0 = split * g.chunks_per_split;
    const int c1 = min(g.n_chunks, c0 + g.chunks_per_split);
    const int nch = max(0, c1 - c0);
    const int N = g.N;
    const uint32_t ncols = uint32_t(2 * N);

    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1 + kEpiWarps);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(&tfull[s], 1);
            mbar_init(&tempty[s], kEpiWarps);
        }
        mbar_init(afull, 1);
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kEpiWarps + 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == kEpiWarps) {
        // ---------------- producer: data tile once, then dictionary chunks ----------------
        if (lane == 0) {
            mbar_expect_tx(afull, a_bytes);
            bulk_g2s(sA, g.a_ops + size_t(tile) * a_bytes, a_bytes, afull);
            int issued = 0;
            for (int i = 0; i < nch; ++i) {
                const int s = i % NS;
                if (i >= NS && !mbar_wait(&empty[s], ((i / NS) - 1) & 1, abort_flag, g.wait_ns)) break;
                ++issued;
                const int c = c0 + i;
                mbar_expect_tx(&full[s], b_bytes + x_bytes);
                bulk_g2s(sB + size_t(s) * b_bytes, g.b_ops + size_t(c) * b_bytes, b_bytes, &full[s]);
                float* xs = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(sX) + size_t(s) * x_bytes);
                bulk_g2s(xs, g.dn + size_t(c) * N, N * 4, &full[s]);
                for (int u = 0; u < g.users; ++u)
                    bulk_g2s(xs + (1 + u) * N, g.aw + size_t(u) * g.Mpad + size_t(c) * N, N * 4, &full[s]);
                bulk_g2s(xs + (1 + g.users) * N, g.fw + size_t(c) * N, N * 4, &full[s]);
                bulk_g2s(xs + (2 + g.users) * N, g.gate + size_t(c) * 4, 16, &full[s]);
            }
            // no bulk copy may still be writing shared memory when the CTA exits
            mbar_drain(afull, 0);
            for (int i = max(0, issued - NS); i < issued; ++i) mbar_drain(&full[i % NS], (i / NS) & 1);
        }
    } else if (warp == kEpiWarps + 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0 && mbar_wait(afull, 0, abort_flag, g.wait_ns)) {
            const uint32_t idesc = instr_desc<MODE>(kTileM, N);
            const uint32_t lbo_a = kTileM * 16, lbo_b = uint32_t(N) * 16;
            const int ksteps = g.Kp / T::kStepK;
            const int lo_off = g.Kp / T::kChunk; // K chunks to the lo half
            for (int i = 0; i < nch; ++i) {
                const int s = i % NS, buf = i & 1;
                if (!mbar_wait(&full[s], (i / NS) & 1, abort_flag, g.wait_ns)) break;
                if (i >= 2 && !mbar_wait(&tempty[buf], ((i >> 1) - 1) & 1, abort_flag, g.wait_ns)) break;
                tc_fence_after();
                const uint8_t* b = sB + size_t(s) * b_bytes;
                const uint32_t d = tmem + uint32_t(buf * N);
                uint32_t acc = 0;
                for (int kk = 0; kk < ksteps; ++kk) {
                    const uint64_t ah = smem_desc(sA + size_t(2 * kk) * lbo_a, lbo_a, 128);
                    const uint64_t bh = smem_desc(b + size_t(2 * kk) * lbo_b, lbo_b, 128);
                    umma<MODE>(d, ah, bh, idesc, acc);
                    acc = 1;
                    if constexpr (T::kSplit) {
                        const uint64_t al = smem_desc(sA + size_t(lo_off + 2 * kk) * lbo_a, lbo_a, 128);
                        const uint64_t bl = smem_desc(b + size_t(lo_off + 2 * kk) * lbo_b, lbo_b, 128);
                        umma<MODE>(d, ah, bl, idesc, 1);
                        umma<MODE>(d, al, bh, idesc, 1);
                    }
                }
                umma_commit(&tfull[buf]); // accumulator ready for the epilogue
                umma_commit(&empty[s]);   // operand stage free once these MMAs completed
            }
        }
        if (lane == 0) {
            // every MMA of this CTA has completed before tensor memory is released
            umma_commit(done);
            mbar_drain(done, 0);
        }
    } else {
        // ---------------- epilogue: 8 warps ----------------
        const int q = warp & 3, h = warp >> 2;
        const int row = tile * kTileM + q * 32 + lane;
        const bool valid = row < g.n_samples;
        const float xn = valid ? g.xn[row] : 0.f;
        const float exn_max = fix_scale<MODE>() > 0.f ? warp_exn_max(g.ewl2, xn) : 0.f;
        float acc[NU];
#pragma unroll
        for (int u = 0; u < NU; ++u) acc[u] = 0.f;
        const int half = N / 2;
        // flagged entries of one batch of columns: exact squared distance from the FP32 rows
        auto fix = [&](uint32_t mask, const float* xs, int col, int c) {
            if (!valid) return;
            while (mask) {
                const int j = __ffs(mask) - 1;
                mask &= mask - 1u;
                const float d2 = row_distance(g.xrows + size_t(row) * g.Dp, g.drows + size_t(c * N + col + j) * g.Dp, g.D);
                const float kv = ex2(g.ewl2 * d2);
#pragma unroll
                for (int u = 0; u < NU; ++u)
                    if (u < g.users) acc[u] = fmaf(xs[(1 + u) * N + col + j], kv, acc[u]);
            }
        };
        for (int i = 0; i < nch; ++i) {
            const int s = i % NS, buf = i & 1;
            // the stage's norms / coefficients (bulk copies) and the accumulator
            if (!mbar_wait(&full[s], (i / NS) & 1, abort_flag, g.wait_ns)) break;
            if (!mbar_wait(&tfull[buf], (i >> 1) & 1, abort_flag, g.wait_ns)) break;
            tc_fence_after();
            const float* xs = reinterpret_cast<const float*>(reinterpret_cast<const uint8_t*>(sX) + size_t(s) * x_bytes);
            const uint32_t trow = tmem + (uint32_t(q * 32) << 16) + uint32_t(buf * N);
            // can any entry of this chunk exceed the bound for a row of this warp?  (warp-uniform)
            const float* gate = xs + (2 + g.users) * N;
            const bool check = fix_scale<MODE>() > 0.f && fmaf(exn_max, gate[0], gate[1]) > 1.f;
            if (half >= 32) {
                for (int cb = 0; cb < half; cb += 32) {
                    const int col = h * half + cb;
                    float gv[32];
                    tmem_ld32(trow + uint32_t(col), gv);
                    if (check) fix(epilogue_columns<32, NU, true>(gv, xs + col, N, xn, g.ewl2, g.users, acc), xs, col, c0 + i);
                    else epilogue_columns<32, NU, false>(gv, xs + col, N, xn, g.ewl2, g.users, acc);
                }
            } else { // 32-column chunks: 16 columns per half
                const int col = h * half;
                float gv[16];
                tmem_ld16(trow + uint32_t(col), gv);
                if (check) fix(epilogue_columns<16, NU, true>(gv, xs + col, N, xn, g.ewl2, g.users, acc), xs, col, c0 + i);
                else epilogue_columns<16, NU, false>(gv, xs + col, N, xn, g.ewl2, g.users, acc);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&tempty[buf]);
                mbar_arrive(&empty[s]);
            }
        }
        // combine the two column halves: warps 4-7 hand their sums to warps 0-3
        asm volatile("bar.sync 1, %0;" ::"r"(kEpiWarps * 32) : "memory");
        if (h == 1) {
#pragma unroll
            for (int u = 0; u < NU; ++u)
                if (u < g.users) red[(q * 32 + lane) * g.users + u] = acc[u];
        }
        asm volatile("bar.sync 1, %0;" ::"r"(kEpiWarps * 32) : "memory");
        if (h == 0 && row < g.n_samples) {
#pragma unroll
            for (int u = 0; u < NU; ++u)
                if (u < g.users)
                    g.part[(size_t(split) * g.users + u) * g.n_samples + row] =
                        acc[u] + red[(q * 32 + lane) * g.users + u];
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == kEpiWarps + 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
    }
    if (threadIdx.x == 0 && *abort_flag) atomicExch(g.err, 1);
}

// out[u][s] = wL <w_u, x_s> + sum_split part[split][u][s] (fixed order).  A block
// takes kFinSamples samples: their rows are read once, coalesced, into shared
// memory, and warp u forms user u's linear terms (lane = sample, d in order).
constexpr int kFinSamples = 32;
constexpr int kFinWarps = 16;

__global__ void __launch_bounds__(kFinWarps * 32)
    gram_finish_kernel(const float* __restrict__ xs, int Dp, int D, const float* __restrict__ w, float wL,
                       const float* __restrict__ part, int splits, int users, int n_samples, float* __restrict__ out,
                       size_t out_stride)
{
    __shared__ float xt[kFinSamples][kMaxFeatures + 1];
    const int s0 = blockIdx.x * kFinSamples;
    for (int idx = threadIdx.x; idx < kFinSamples * D; idx += kFinWarps * 32) {
        const int r = idx / D, d = idx % D;
        xt[r][d] = s0 + r < n_samples ? xs[size_t(s0 + r) * Dp + d] : 0.f;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, s = s0 + lane;
    for (int u = threadIdx.x >> 5; u < users; u += kFinWarps) {
        const float* wu = w + size_t(u) * D;
        float lin = 0.f;
        for (int d = 0; d < D; ++d) lin = fmaf(__ldg(wu + d), xt[lane][d], lin);
        if (s < n_samples) {
            float gsum = 0.f;
            for (int sp = 0; sp < splits; ++sp) gsum += part[(size_t(sp) * users + u) * n_samples + s];
            out[size_t(u) * out_stride + s] = fmaf(wL, lin, gsum);
        }
    }
}

// ------------------------------------------------ two-product form (users >= 4) --
// The users' contraction on the tensor cores too: per chunk of N dictionary
// rows, the epilogue turns the Gram tile into kernel values P (128 x N, in the
// mode's operand format: hi [+ lo]) in shared memory, and a second UMMA
// (M = 128, N = 16 users, K = N rows) accumulates P W with W the chunk's
// coefficients a * wG (16 x N, padded with zero users) into tensor memory for
// the whole dictionary range of the CTA.  The epilogue then costs one
// exponential and a store per kernel value instead of one FMA per user; the
// second product rounds P and W to the operand format (split modes: hi/lo, 3
// products).  Used for the BF16 form with 4 or more users: at N = 64, 16
// users, a 65536-symbol detection takes 1.66 ms instead of 3.21 ms, the soft
// outputs moving from 1.4e-6 to 5.2e-5 of the largest output away from the
// float64 model (decisions unchanged); the TF32 form gains 2 % for a 10x
// larger error and the split forms lose time (larger P buffers, 3 products),
// so they keep the one-product kernel.
constexpr int kUsers2 = 16; // UMMA N of the users' product

struct Gram2Args {
    const uint8_t* a_ops; // data tiles (kTileM rows)
    const uint8_t* b_ops; // dictionary chunks (N rows)
    const uint8_t* w_ops; // per chunk: W, 16 rows x N (K), canonical K-major, hi [| lo]
    const float* xn;      // data norms
    const float* dn;      // dictionary norms (Mpad)
    const float* fw;      // fix weights (Mpad)
    const float* gate;    // per chunk: max fw, max fw |ewl2 dn|, 0, 0
    const float* xrows;   // data rows (n_samples x Dp, FP32) for the exact recompute
    const float* drows;   // dictionary rows (M x Dp, FP32)
    float* part;          // splits x users x n_samples partial sums
    int* err;
    int n_samples, users, Kp, N, Dp, D;
    int chunks_per_split, n_chunks;
    int stages;
    float ewl2; // ew * log2(e)
    unsigned long long wait_ns; // limit of the bounded waits
};

// 16 kernel values of one data row (columns col .. col + 15 of the chunk) into the
// kernel-value operand P (row r; hi [and lo]).  CHECK: entries whose error bound
// exceeds kFixEps are returned as bits of the mask (their P entries are rewritten).
template <int MODE, bool CHECK>
__device__ __forceinline__ uint32_t kernel_values16(const float* gv, const float* sd, int N, int col, float xn,
                                                    float ewl2, uint8_t* p, int r)
{
    using T = OpTraits<MODE>;
    uint32_t mask = 0u;
#pragma unroll
    for (int j0 = 0; j0 < 16; j0 += T::kChunk) {
        // one 16-byte K chunk of this row: hi, and lo for split modes
        uint32_t hw[4] = {0u, 0u, 0u, 0u}, lw[4] = {0u, 0u, 0u, 0u};
        float kv[T::kChunk];
#pragma unroll
        for (int e = 0; e < T::kChunk; ++e) {
            const int j = j0 + e;
            const float t = xn + sd[col + j];
            kv[e] = ex2(ewl2 * fmaxf(fmaf(-2.f, gv[j], t), 0.f));
            if constexpr (CHECK)
                if (kv[e] * (ewl2 * t) * sd[N + col + j] < -1.f) mask |= 1u << j;
        }
        if constexpr (MODE == kBF16) {
            // pairs converted by one instruction each (round to nearest)
#pragma unroll
            for (int e = 0; e < T::kChunk; e += 2) {
                const __nv_bfloat162 v2 = __floats2bfloat162_rn(kv[e], kv[e + 1]);
                hw[e >> 1] = *reinterpret_cast<const uint32_t*>(&v2);
            }
        } else {
#pragma unroll
            for (int e = 0; e < T::kChunk; ++e) {
                float hi, lo;
                split_operand<MODE>(kv[e], &hi, &lo);
                if constexpr (T::kTF) {
                    hw[e] = __float_as_uint(hi);
                    lw[e] = __float_as_uint(lo);
                } else {
                    hw[e >> 1] |= uint32_t(__bfloat16_as_ushort(__float2bfloat16_rn(hi))) << (16 * (e & 1));
                    lw[e >> 1] |= uint32_t(__bfloat16_as_ushort(__float2bfloat16_rn(lo))) << (16 * (e & 1));
                }
            }
        }
        const int kc = (col + j0) / T::kChunk;
        const size_t off = size_t(kc) * (kTileM * 16) + (r >> 3) * 128 + (r & 7) * 16;
        *reinterpret_cast<uint4*>(p + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        if constexpr (T::kSplit)
            *reinterpret_cast<uint4*>(p + size_t(N / T::kChunk) * (kTileM * 16) + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
    return mask;
}

// W chunks: element (u, k) = a[u][c N + k] * wG (0 past M and for u >= users)
template <int MODE>
__global__ void gram_pack_w_kernel(const float* __restrict__ a, size_t a_stride, int users, int M, int N, int n_chunks,
                                   float wG, uint8_t* __restrict__ w_ops)
{
    using T = OpTraits<MODE>;
    const int KE2 = T::kSplit ? 2 * N : N;
    const size_t total = size_t(n_chunks) * kUsers2 * N;
    for (size_t idx = blockIdx.x * size_t(blockDim.x) + threadIdx.x; idx < total; idx += size_t(gridDim.x) * blockDim.x) {
        const int k = int(idx % N);
        const size_t rest = idx / N;
        const int u = int(rest % kUsers2), c = int(rest / kUsers2);
        const int b = c * N + k;
        const float v = (u < users && b < M) ? __fmul_rn(a[size_t(u) * a_stride + b], wG) : 0.f;
        float hi, lo;
        split_operand<MODE>(v, &hi, &lo);
        uint8_t* tile = w_ops + size_t(c) * kUsers2 * KE2 * T::kElem;
        put_operand<MODE>(tile, kUsers2, u, k, hi);
        if constexpr (T::kSplit) put_operand<MODE>(tile, kUsers2, u, N + k, lo);
    }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, 1) gram_detect2_kernel(Gram2Args g)
{
    using T = OpTraits<MODE>;
    extern __shared__ __align__(1024) uint8_t smem[];
    const int N = g.N, NS = g.stages;
    const int KE = T::kSplit ? 2 * g.Kp : g.Kp;
    const int KE2 = T::kSplit ? 2 * N : N; // K extent of the second product's operands
    const uint32_t a_bytes = uint32_t(kTileM) * KE * T::kElem;
    const uint32_t b_bytes = uint32_t(N) * KE * T::kElem;
    const uint32_t w_bytes = uint32_t(kUsers2) * KE2 * T::kElem;
    const uint32_t p_bytes = uint32_t(kTileM) * KE2 * T::kElem;
    uint8_t* sA = smem;
    uint8_t* sB = sA + a_bytes;                          // [NS] chunk rows
    uint8_t* sW = sB + size_t(NS) * b_bytes;             // [NS] chunk coefficients
    uint8_t* sP = sW + size_t(NS) * w_bytes;             // [2] kernel values
    const int sd_stride = 2 * N + 4;                     // chunk norms, fix weights, gate
    float* sD = reinterpret_cast<float*>(sP + 2 * size_t(p_bytes)); // [NS][sd_stride]
    uint64_t* bars = reinterpret_cast<uint64_t*>(sD + size_t(NS) * sd_stride);
    uint64_t* full = bars;             // [NS]
    uint64_t* empty = bars + NS;       // [NS]
    uint64_t* tfull = bars + 2 * NS;   // [2]
    uint64_t* tempty = tfull + 2;      // [2]
    uint64_t* pfull = tempty + 2;      // [2]
    uint64_t* pempty = pfull + 2;      // [2]
    uint64_t* afull = pempty + 2;      // [1]
    uint64_t* done = afull + 1;        // [1] every product of the CTA completed
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x, split = blockIdx.y;
    const int c0 = split * g.chunks_per_split;
    const int c1 = min(g.n_chunks, c0 + g.chunks_per_split);
    const int nch = max(0, c1 - c0);
    uint32_t ncols = 32;
    while (ncols < uint32_t(2 * N + kUsers2)) ncols <<= 1;
    const uint32_t acc2 = uint32_t(2 * N); // column of the users' accumulator

    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1 + kEpiWarps);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(&tfull[s], 1);
            mbar_init(&tempty[s], kEpiWarps);
            mbar_init(&pfull[s], kEpiWarps);
            mbar_init(&pempty[s], 1);
        }
        mbar_init(afull, 1);
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kEpiWarps + 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == kEpiWarps) {
        // ---------------- producer: data tile once, then dictionary chunks with their W and norms ----------------
        if (lane == 0) {
            mbar_expect_tx(afull, a_bytes);
            bulk_g2s(sA, g.a_ops + size_t(tile) * a_bytes, a_bytes, afull);
            int issued = 0;
            for (int i = 0; i < nch; ++i) {
                const int s = i % NS;
                if (i >= NS && !mbar_wait(&empty[s], ((i / NS) - 1) & 1, abort_flag, g.wait_ns)) break;
                ++issued;
                const int c = c0 + i;
                mbar_expect_tx(&full[s], b_bytes + w_bytes + uint32_t(sd_stride) * 4);
                bulk_g2s(sB + size_t(s) * b_bytes, g.b_ops + size_t(c) * b_bytes, b_bytes, &full[s]);
                bulk_g2s(sW + size_t(s) * w_bytes, g.w_ops + size_t(c) * w_bytes, w_bytes, &full[s]);
                float* sd = sD + size_t(s) * sd_stride;
                bulk_g2s(sd, g.dn + size_t(c) * N, uint32_t(N) * 4, &full[s]);
                bulk_g2s(sd + N, g.fw + size_t(c) * N, uint32_t(N) * 4, &full[s]);
                bulk_g2s(sd + 2 * N, g.gate + size_t(c) * 4, 16, &full[s]);
            }
            mbar_drain(afull, 0);
            for (int i = max(0, issued - NS); i < issued; ++i) mbar_drain(&full[i % NS], (i / NS) & 1);
        }
    } else if (warp == kEpiWarps + 1) {
        // ---------------- MMA issuer: Gram tile of chunk i, then the users' product of chunk i - 1 ----------------
        if (lane == 0 && mbar_wait(afull, 0, abort_flag, g.wait_ns)) {
            const uint32_t idesc = instr_desc<MODE>(kTileM, N);
            const uint32_t idesc2 = instr_desc<MODE>(kTileM, kUsers2);
            const uint32_t lbo_a = kTileM * 16, lbo_b = uint32_t(N) * 16, lbo_w = kUsers2 * 16;
            const int ksteps = g.Kp / T::kStepK, ksteps2 = N / T::kStepK;
            const int lo_off = g.Kp / T::kChunk, lo_off2 = N / T::kChunk;
            bool ok = true;
            auto product2 = [&](int j) {
                const int pb = j & 1, sj = j % NS;
                if (!mbar_wait(&pfull[pb], (j >> 1) & 1, abort_flag, g.wait_ns)) {
                    ok = false;
                    return;
                }
                tc_fence_after();
                const uint8_t* p = sP + size_t(pb) * p_bytes;
                const uint8_t* w = sW + size_t(sj) * w_bytes;
                for (int kk = 0; kk < ksteps2; ++kk) {
                    const uint64_t ah = smem_desc(p + size_t(2 * kk) * lbo_a, lbo_a, 128);
                    const uint64_t bh = smem_desc(w + size_t(2 * kk) * lbo_w, lbo_w, 128);
                    umma<MODE>(tmem + acc2, ah, bh, idesc2, (j > 0 || kk > 0) ? 1u : 0u);
                    if constexpr (T::kSplit) {
                        const uint64_t al = smem_desc(p + size_t(lo_off2 + 2 * kk) * lbo_a, lbo_a, 128);
                        const uint64_t bl = smem_desc(w + size_t(lo_off2 + 2 * kk) * lbo_w, lbo_w, 128);
                        umma<MODE>(tmem + acc2, ah, bl, idesc2, 1u);
                        umma<MODE>(tmem + acc2, al, bh, idesc2, 1u);
                    }
                }
                umma_commit(&pempty[pb]); // kernel-value buffer free once these products completed
                umma_commit(&empty[sj]);  // the chunk's rows and coefficients too
            };
            for (int i = 0; i < nch && ok; ++i) {
                const int s = i % NS, buf = i & 1;
                if (!mbar_wait(&full[s], (i / NS) & 1, abort_flag, g.wait_ns)) break;
                if (i >= 2 && !mbar_wait(&tempty[buf], ((i >> 1) - 1) & 1, abort_flag, g.wait_ns)) break;
                tc_fence_after();
                const uint8_t* b = sB + size_t(s) * b_bytes;
                const uint32_t d = tmem + uint32_t(buf * N);
                for (int kk = 0; kk < ksteps; ++kk) {
                    const uint64_t ah = smem_desc(sA + size_t(2 * kk) * lbo_a, lbo_a, 128);
                    const uint64_t bh = smem_desc(b + size_t(2 * kk) * lbo_b, lbo_b, 128);
                    umma<MODE>(d, ah, bh, idesc, kk > 0 ? 1u : 0u);
                    if constexpr (T::kSplit) {
                        const uint64_t al = smem_desc(sA + size_t(lo_off + 2 * kk) * lbo_a, lbo_a, 128);
                        const uint64_t bl = smem_desc(b + size_t(lo_off + 2 * kk) * lbo_b, lbo_b, 128);
                        umma<MODE>(d, ah, bl, idesc, 1);
                        umma<MODE>(d, al, bh, idesc, 1);
                    }
                }
                umma_commit(&tfull[buf]); // Gram tile ready for the epilogue
                if (i >= 1) product2(i - 1);
            }
            if (ok && nch > 0 && !*abort_flag) product2(nch - 1);
        }
        if (lane == 0) {
            umma_commit(done);
            mbar_drain(done, 0);
        }
    } else {
        // ---------------- epilogue: kernel values of each chunk into P; at the end the users' sums ----------------
        const int q = warp & 3, h = warp >> 2;
        const int r = q * 32 + lane; // row of the tile (tensor-memory lane)
        const int row = tile * kTileM + r;
        const bool valid = row < g.n_samples;
        const float xn = valid ? g.xn[row] : 0.f;
        constexpr bool kFix = fix_scale<MODE>() > 0.f && !T::kSplit;
        const float exn_max = kFix ? warp_exn_max(g.ewl2, xn) : 0.f;
        const int half = N / 2;
        bool ok = true;
        for (int i = 0; i < nch; ++i) {
            const int s = i % NS, buf = i & 1, pb = i & 1;
            if (!mbar_wait(&full[s], (i / NS) & 1, abort_flag, g.wait_ns) ||
                !mbar_wait(&tfull[buf], (i >> 1) & 1, abort_flag, g.wait_ns) ||
                (i >= 2 && !mbar_wait(&pempty[pb], ((i >> 1) - 1) & 1, abort_flag, g.wait_ns))) {
                ok = false;
                break;
            }
            tc_fence_after();
            const float* sd = sD + size_t(s) * sd_stride;
            uint8_t* p = sP + size_t(pb) * p_bytes;
            const uint32_t trow = tmem + (uint32_t(q * 32) << 16) + uint32_t(buf * N);
            // can any entry of this chunk exceed the bound for a row of this warp?  (warp-uniform)
            const bool check = kFix && fmaf(exn_max, sd[2 * N], sd[2 * N + 1]) > 1.f;
            for (int cb = 0; cb < half; cb += 16) {
                const int col = h * half + cb;
                float gv[16];
                tmem_ld16(trow + uint32_t(col), gv);
                if (!check) {
                    kernel_values16<MODE, false>(gv, sd, N, col, xn, g.ewl2, p, r);
                    continue;
                }
                uint32_t mask = kernel_values16<MODE, true>(gv, sd, N, col, xn, g.ewl2, p, r);
                if (!valid) mask = 0u;
                // flagged entries: exact squared distance from the FP32 rows, the value rewritten in P
                while (mask) {
                    const int j = __ffs(mask) - 1;
                    mask &= mask - 1u;
                    const float d2 = row_distance(g.xrows + size_t(row) * g.Dp,
                                                  g.drows + size_t((c0 + i) * N + col + j) * g.Dp, g.D);
                    put_operand<MODE>(p, kTileM, r, col + j, ex2(g.ewl2 * d2));
                }
            }
            tc_fence_before();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); // P visible to the tensor cores
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&tempty[buf]);
                mbar_arrive(&empty[s]);
                mbar_arrive(&pfull[pb]);
            }
        }
        if (h == 0) {
            // warps 0-3 read the users' sums of their 32 lanes (tcgen05.ld is warp-wide: the
            // whole warp loads, the lanes of rows past the end discard)
            float acc[kUsers2];
#pragma unroll
            for (int u = 0; u < kUsers2; ++u) acc[u] = 0.f;
            const bool have = ok && nch > 0 && mbar_wait(done, 0, abort_flag, g.wait_ns);
            if (__all_sync(0xffffffffu, have)) {
                tc_fence_after();
                tmem_ld16(tmem + (uint32_t(q * 32) << 16) + acc2, acc);
            }
            if (row < g.n_samples)
                for (int u = 0; u < g.users; ++u) g.part[(size_t(split) * g.users + u) * g.n_samples + row] = acc[u];
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == kEpiWarps + 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
    }
    if (threadIdx.x == 0 && *abort_flag) atomicExch(g.err, 1);
}

template <int MODE> size_t gram2_smem(int Kp, int N, int stages)
{
    using T = OpTraits<MODE>;
    const size_t KE = T::kSplit ? 2 * Kp : Kp, KE2 = T::kSplit ? 2 * N : N;
    return size_t(kTileM) * KE * T::kElem + size_t(stages) * (size_t(N) * KE * T::kElem + kUsers2 * KE2 * T::kElem) +
           2 * size_t(kTileM) * KE2 * T::kElem + size_t(stages) * (2 * N + 4) * 4 + (2 * stages + 10) * 8 + 16;
}

template <int MODE, int NU> void launch_gram(const GramArgs& ga, int n_tiles, int splits, size_t smem, cudaStream_t s,
                                             cudaError_t* e)
{
    *e = cudaFuncSetAttribute(gram_detect_kernel<MODE, NU>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (*e != cudaSuccess) return;
    gram_detect_kernel<MODE, NU><<<dim3(n_tiles, splits), kThreads, smem, s>>>(ga);
    *e = cudaGetLastError();
}

template <int MODE>
apsm_status run_gram2(apsm_detector* h, uint32_t S, float* d_out, cudaStream_t s, int Kp, int N, int stages)
{
    using T = OpTraits<MODE>;
    if (2 * N + kUsers2 > 512) { // the kernel's tensor memory: 2 N + 16 columns rounded up to a power of two
        h->last_error = "two-product Gram detection: chunk of " + std::to_string(N) + " rows exceeds tensor memory";
        return APSM_ERR_UNSUPPORTED;
    }
    GramWorkspace* gw = h->gram;
    const int ns = int(2 * S);
    const int M = int(h->used);
    const int D = int(h->D), Dp = int(h->Dp), U = int(h->U);
    const int KE = T::kSplit ? 2 * Kp : Kp, KE2 = T::kSplit ? 2 * N : N;
    const int n_tiles = (ns + kTileM - 1) / kTileM;
    const int n_chunks = std::max(1, (M + N - 1) / N);
    const int Mpad = n_chunks * N;
    int splits = std::max(1, std::min(n_chunks, (148 + n_tiles - 1) / n_tiles)); // one CTA per SM
    const int cps = (n_chunks + splits - 1) / splits;
    splits = (n_chunks + cps - 1) / cps;

    cudaError_t e;
#define GR_CK(x)                                                   \
    do {                                                           \
        e = (x);                                                   \
        if (e != cudaSuccess) return h->cuda_fail(e, #x);          \
    } while (0)
    GR_CK(gw->a_ops.ensure(size_t(n_tiles) * kTileM * KE * T::kElem));
    GR_CK(gw->b_ops.ensure(size_t(n_chunks) * N * KE * T::kElem));
    GR_CK(gw->w_ops.ensure(size_t(n_chunks) * kUsers2 * KE2 * T::kElem));
    GR_CK(gw->xn.ensure(size_t(n_tiles) * kTileM));
    GR_CK(gw->dn.ensure(Mpad));
    GR_CK(gw->fw.ensure(Mpad));
    GR_CK(gw->gate.ensure(size_t(4) * n_chunks));
    GR_CK(gw->part.ensure(size_t(splits) * U * ns));
    GR_CK(gw->err.ensure(1));
    GR_CK(cudaMemsetAsync(gw->err.p, 0, sizeof(int), s));
    GR_CK(cudaMemsetAsync(gw->dn.p, 0, sizeof(float) * Mpad, s));
    const float ewl2 = h->model_params().ew * 1.4426950408889634f;

    const int threads = 256;
    gram_pack_kernel<MODE><<<std::min(4096, (n_tiles * kTileM * Kp + threads - 1) / threads), threads, 0, s>>>(
        h->xs.p, ns, Dp, D, Kp, kTileM, n_tiles, gw->a_ops.p, gw->xn.p);
    GR_CK(cudaGetLastError());
    gram_pack_kernel<MODE><<<std::min(4096, (n_chunks * N * Kp + threads - 1) / threads), threads, 0, s>>>(
        h->dict_X.p, M, Dp, D, Kp, N, n_chunks, gw->b_ops.p, gw->dn.p);
    GR_CK(cudaGetLastError());
    gram_fix_kernel<MODE><<<n_chunks, 256, 0, s>>>(h->dict_a.p, h->cap, U, M, N, h->cfg.wG, ewl2, gw->dn.p, gw->fw.p,
                                                   gw->gate.p);
    GR_CK(cudaGetLastError());
    gram_pack_w_kernel<MODE><<<std::min(4096, (n_chunks * kUsers2 * N + threads - 1) / threads), threads, 0, s>>>(
        h->dict_a.p, h->cap, U, M, N, n_chunks, h->cfg.wG, gw->w_ops.p);
    GR_CK(cudaGetLastError());

    Gram2Args ga;
    ga.a_ops = gw->a_ops.p;
    ga.b_ops = gw->b_ops.p;
    ga.w_ops = gw->w_ops.p;
    ga.xn = gw->xn.p;
    ga.dn = gw->dn.p;
    ga.fw = gw->fw.p;
    ga.gate = gw->gate.p;
    ga.xrows = h->xs.p;
    ga.drows = h->dict_X.p;
    ga.part = gw->part.p;
    ga.err = gw->err.p;
    ga.n_samples = ns;
    ga.users = U;
    ga.Kp = Kp;
    ga.N = N;
    ga.Dp = Dp;
    ga.D = D;
    ga.chunks_per_split = cps;
    ga.n_chunks = n_chunks;
    ga.stages = stages;
    ga.ewl2 = ewl2;
    ga.wait_ns = wait_limit_ns();
    // >= 120 KB keeps one CTA per SM: its tensor memory (up to 512 columns) is never contended
    const size_t smem = std::max<size_t>(gram2_smem<MODE>(Kp, N, stages) + 1024, 120 * 1024);
    GR_CK(cudaFuncSetAttribute(gram_detect2_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    gram_detect2_kernel<MODE><<<dim3(n_tiles, splits), kThreads, smem, s>>>(ga);
    GR_CK(cudaGetLastError());
    gram_finish_kernel<<<(ns + kFinSamples - 1) / kFinSamples, kFinWarps * 32, 0, s>>>(
        h->xs.p, Dp, D, h->w.p, h->cfg.wL, gw->part.p, splits, U, ns, d_out, size_t(ns));
    GR_CK(cudaGetLastError());
    GR_CK(cudaMemcpyAsync(gw->h_err, gw->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
#undef GR_CK
    return APSM_OK;
}

template <int MODE>
apsm_status run_gram(apsm_detector* h, uint32_t S, float* d_out, cudaStream_t s)
{
    using T = OpTraits<MODE>;
    GramWorkspace* gw = h->gram;
    const int ns = int(2 * S);
    const int M = int(h->used);
    const int D = int(h->D), Dp = int(h->Dp), U = int(h->U);
    if (U > kMaxUsers) {
        h->last_error = "Gram detection supports at most " + std::to_string(kMaxUsers) + " users per detector";
        return APSM_ERR_UNSUPPORTED;
    }
    const int Kp = int(round_up(uint32_t(D), uint32_t(T::kStepK)));
    const int KE = T::kSplit ? 2 * Kp : Kp;
    if (MODE == kBF16 && U >= 4 && !h->gram_one_product) {
        // the users' contraction on the tensor cores where its operands fit shared memory; only
        // in the BF16 form, whose kernel values and coefficients may be BF16 too (in the other
        // forms the second product's rounding would cost more accuracy than its time saves)
        // tensor memory: two Gram buffers of n2 columns and the users' 16, rounded up to a power of
        // two, within the 512 columns of an SM: n2 <= 128
        for (int n2 = 128; n2 >= 32; n2 /= 2)
            for (int st2 = kMaxStages; st2 >= 2; --st2)
                if (gram2_smem<MODE>(Kp, n2, st2) + 1024 <= 220 * 1024) return run_gram2<MODE>(h, S, d_out, s, Kp, n2, st2);
    }
    // dictionary chunk width and stages: the data tile and the chunk ring within shared memory
    // (chunks of 256 down to 64 columns in 3 stages, then 32 columns in 3 or 2 stages)
    int N = 256, stages = kMaxStages;
    auto smem_for = [&](int n, int st) {
        return size_t(kTileM) * KE * T::kElem + size_t(st) * (size_t(n) * KE * T::kElem + size_t(n) * 4 * (2 + U) + 16) +
               (2 * st + 6) * 8 + 16 + size_t(4 * 32) * U * 4;
    };
    const size_t limit = 220 * 1024;
    while (N > 32 && smem_for(N, stages) > limit) N /= 2;
    if (smem_for(N, stages) > limit) stages = 2;
    if (smem_for(N, stages) > limit) {
        h->last_error = "Gram detection operands do not fit shared memory";
        return APSM_ERR_UNSUPPORTED;
    }
    const int n_tiles = (ns + kTileM - 1) / kTileM;
    const int n_chunks = std::max(1, (M + N - 1) / N);
    const int Mpad = n_chunks * N;
    int splits = std::max(1, std::min(n_chunks, (2 * 148 + n_tiles - 1) / n_tiles));
    const int cps = (n_chunks + splits - 1) / splits;
    splits = (n_chunks + cps - 1) / cps;

    cudaError_t e;
#define GR_CK(x)                                                   \
    do {                                                           \
        e = (x);                                                   \
        if (e != cudaSuccess) return h->cuda_fail(e, #x);          \
    } while (0)
    GR_CK(gw->a_ops.ensure(size_t(n_tiles) * kTileM * KE * T::kElem));
    GR_CK(gw->b_ops.ensure(size_t(n_chunks) * N * KE * T::kElem));
    GR_CK(gw->xn.ensure(size_t(n_tiles) * kTileM));
    GR_CK(gw->dn.ensure(Mpad));
    GR_CK(gw->aw.ensure(size_t(U) * Mpad));
    GR_CK(gw->fw.ensure(Mpad));
    GR_CK(gw->gate.ensure(size_t(4) * n_chunks));
    GR_CK(gw->part.ensure(size_t(splits) * U * ns));
    GR_CK(gw->err.ensure(1));
    GR_CK(cudaMemsetAsync(gw->err.p, 0, sizeof(int), s));
    GR_CK(cudaMemsetAsync(gw->dn.p, 0, sizeof(float) * Mpad, s));
    const float ewl2 = h->model_params().ew * 1.4426950408889634f;

    const int threads = 256;
    gram_pack_kernel<MODE><<<std::min(4096, (n_tiles * kTileM * Kp + threads - 1) / threads), threads, 0, s>>>(
        h->xs.p, ns, Dp, D, Kp, kTileM, n_tiles, gw->a_ops.p, gw->xn.p);
    GR_CK(cudaGetLastError());
    gram_pack_kernel<MODE><<<std::min(4096, (n_chunks * N * Kp + threads - 1) / threads), threads, 0, s>>>(
        h->dict_X.p, M, Dp, D, Kp, N, n_chunks, gw->b_ops.p, gw->dn.p);
    GR_CK(cudaGetLastError());
    gram_coeff_kernel<<<(U * Mpad + 255) / 256, 256, 0, s>>>(h->dict_a.p, h->cap, U, M, Mpad, h->cfg.wG, gw->aw.p);
    GR_CK(cudaGetLastError());
    gram_fix_kernel<MODE><<<n_chunks, 256, 0, s>>>(h->dict_a.p, h->cap, U, M, N, h->cfg.wG, ewl2, gw->dn.p, gw->fw.p,
                                                   gw->gate.p);
    GR_CK(cudaGetLastError());

    GramArgs ga;
    ga.a_ops = gw->a_ops.p;
    ga.b_ops = gw->b_ops.p;
    ga.xn = gw->xn.p;
    ga.dn = gw->dn.p;
    ga.aw = gw->aw.p;
    ga.fw = gw->fw.p;
    ga.gate = gw->gate.p;
    ga.xrows = h->xs.p;
    ga.drows = h->dict_X.p;
    ga.part = gw->part.p;
    ga.err = gw->err.p;
    ga.n_samples = ns;
    ga.Mpad = Mpad;
    ga.users = U;
    ga.Kp = Kp;
    ga.N = N;
    ga.Dp = Dp;
    ga.D = D;
    ga.chunks_per_split = cps;
    ga.n_chunks = n_chunks;
    ga.stages = stages;
    ga.ewl2 = ewl2;
    ga.wait_ns = wait_limit_ns();
    // >= 120 KB keeps one CTA per SM, so the 2N tensor-memory columns of a CTA never wait for another's
    const size_t smem = std::max<size_t>(smem_for(N, stages) + 1024, 120 * 1024);
    if (U <= 1) launch_gram<MODE, 1>(ga, n_tiles, splits, smem, s, &e);
    else if (U <= 2) launch_gram<MODE, 2>(ga, n_tiles, splits, smem, s, &e);
    else if (U <= 4) launch_gram<MODE, 4>(ga, n_tiles, splits, smem, s, &e);
    else if (U <= 8) launch_gram<MODE, 8>(ga, n_tiles, splits, smem, s, &e);
    else launch_gram<MODE, 16>(ga, n_tiles, splits, smem, s, &e);
    if (e != cudaSuccess) return h->cuda_fail(e, "gram_detect_kernel launch");
    gram_finish_kernel<<<(ns + kFinSamples - 1) / kFinSamples, kFinWarps * 32, 0, s>>>(h->xs.p, Dp, D, h->w.p, h->cfg.wL, gw->part.p, splits, U,
                                                            ns, d_out, size_t(ns));
    GR_CK(cudaGetLastError());
    GR_CK(cudaMemcpyAsync(gw->h_err, gw->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
#undef GR_CK
    return APSM_OK;
}

} // namespace
} // namespace apsm

using namespace apsm;

// Expiry of a bounded wait in the last Gram detection, read after its stream
// synchronised (host calls): reported once, then cleared.
apsm_status detect_gram_check(apsm_detector* h)
{
    if (!h->gram || !h->gram->h_err || !*h->gram->h_err) return APSM_OK;
    *h->gram->h_err = 0;
    h->last_error = "Gram detection gave up waiting on the GPU (bounded wait expired); its estimates are invalid";
    return APSM_ERR_CUDA;
}

apsm_status detect_gram(apsm_detector* h, uint32_t S, float* d_out, cudaStream_t s)
{
    if (!h->gram) {
        h->gram = new GramWorkspace();
        if (cudaMallocHost(&h->gram->h_err, sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            h->last_error = "pinned allocation failed";
            return APSM_ERR_OUT_OF_MEMORY;
        }
        *h->gram->h_err = 0;
    }
    if (*h->gram->h_err) { // an earlier call on this stream (device mode) gave up: reported once
        *h->gram->h_err = 0;
        h->last_error = "a previous Gram detection gave up waiting on the GPU (bounded wait expired)";
        return APSM_ERR_CUDA;
    }
    switch (h->cfg.detect_mode) {
    case DetectMode::GramBF16: return run_gram<kBF16>(h, S, d_out, s);
    case DetectMode::GramBF16x3: return run_gram<kBF16x3>(h, S, d_out, s);
    case DetectMode::GramTF32: return run_gram<kTF32>(h, S, d_out, s);
    case DetectMode::GramTF32x3: return run_gram<kTF32x3>(h, S, d_out, s);
    default: break;
    }
    h->last_error = "not a Gram detection mode";
    return APSM_ERR_INVALID_ARGUMENT;
}
