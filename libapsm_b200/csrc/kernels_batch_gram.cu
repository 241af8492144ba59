// Batched tensor-core detection in pair form (tcgen05).  Operands in one of
// the four Gram forms of the single detector: BF16 or TF32 (one UMMA per K
// step), or split hi + lo (three UMMAs per K step: bf16x3 ~2^-16 relative,
// tf32x3 FP32-accurate Gram products).
//
// For data sample s and dictionary pair b (complex y_b) the detector needs
// r = Re(y_b^H x_s) and m = Im(y_b^H x_s) (kernel values of the four row
// combinations, see apsm_batch.cuh).  With A = the samples' rows [Re x; Im x]
// and B = two rows per dictionary pair, [Re y; Im y] and [-Im y; Re y], the
// product A B^T holds r and m in adjacent columns.  One CTA takes a tile of
// 128 samples of one job against every chunk of 64 dictionary pairs
// (UMMA M=128, N=128, FP32 accumulators in tensor memory, double-buffered;
// for the TF32 split form above 32 features, chunks of 32 pairs, N=64, with
// the sample tile in tensor memory: two CTAs per SM instead of one);
// the epilogue forms the three distances with FP32 norms, exponentiates on
// the SFU and accumulates a_2b K(2b, .) + a_2b+1 K(2b+1, .) for the two soft
// outputs of the sample (reference model cpp/lib/apsm/apsm_detect.cu:690-876).
//
// Roles (320 threads): warps 0-7 epilogue (warp w: TMEM lanes 32*(w%4)..,
// column half w/4), warp 8 producer (bulk async copies of the sample tile and
// the dictionary chunks), warp 9 TMEM allocator and MMA issuer.  Every
// mbarrier wait is bounded; on expiry the CTA records an error, still waits
// for its own copies and MMAs, releases tensor memory and returns.
//
// Compensated cross terms (single-product forms bf16 / tf32).  Rounding both
// operands to the format's unit u perturbs r and m by at most 2u |x||y|, so a
// base-2 exponent es + m2 r (es = ew log2(e) (|x|^2 + |y|^2) <= 0) moves by at
// most 2u |es| and the pair's contribution to the two soft outputs by at most
//   (|a_2b| + |a_2b+1|) wG * max(kA, kP, kM) * ln 2 * 2u |es|.
// Where cancellation bites (near-duplicate points: r ~ (|x|^2 + |y|^2) / 2,
// kernel values near 1) that bound is large; the epilogue flags every pair
// whose bound exceeds kFixEps, leaves it out of the tensor-core sums and adds
// it back with r and m recomputed exactly in FP32 from the samples.  Per pair
// the chunk data carries fw = (|a_2b| + |a_2b+1|) wG ln2 2u / kFixEps, and per
// chunk max fw and max fw |ew2 |y|^2|, so a warp whose samples cannot flag any
// pair of a chunk (kernel value <= 1) skips the test.
#include "apsm_batch.cuh"
#include "apsm_tc.cuh"

#include <algorithm>

namespace apsm {

namespace {

using namespace tc;

constexpr int kTileM = 128;      // samples per tile (UMMA M)
constexpr int kEpiWarps = 8;
constexpr int kThreads = (kEpiWarps + 2) * 32;

// Dictionary chunk of CN accumulator columns (UMMA N; two per pair) and its data: a*wG (CN, column
// order), ew log2(e) * pair norms (CN/2), fix weights fw (CN/2), then max fw and
// max fw * |ew log2(e) * pair norm| (padded to 4).  CN = 128, or 64 for the TF32 split form above
// 32 features, whose sample tile then lives in tensor memory so that two CTAs share an SM.
template <int CN> struct Chunk {
    static constexpr int kN = CN;
    static constexpr int kPairs = CN / 2;
    static constexpr int kAw = 0, kNrm = CN, kFw = CN + CN / 2, kGate = 2 * CN;
    static constexpr int kBx = 2 * CN + 4;
    static constexpr bool kAtm = CN == 64; // sample tile in tensor memory
};
__host__ __device__ constexpr int chunk_cols(int mode, int Kp) { return (mode == kTF32x3 && Kp > 32) ? 64 : 128; }
// chunk data ring: the epilogue releases a chunk's data on its own, so an operand stage is free again
// as soon as its products are done (the epilogue never reads the operands)
constexpr int kXRing = 4;
// per-pair error a flagged pair would exceed (soft-output units) in the single-product forms
constexpr float kFixEps = 1.0f / 8192.0f;

// ln 2 * 2u / kFixEps of a mode's operand rounding unit u (0: split forms, no correction)
template <int MODE> __host__ __device__ constexpr float fix_scale()
{
    return MODE == kBF16 ? 0.69314718f * (2.0f / 256.0f) / kFixEps
                         : (MODE == kTF32 ? 0.69314718f * (2.0f / 2048.0f) / kFixEps : 0.0f);
}

// bytes of one operand tile of R rows at K extent Kp (hi [+ lo])
template <int MODE> __host__ __device__ constexpr size_t tile_bytes(int R, int Kp)
{
    return size_t(R) * (OpTraits<MODE>::kSplit ? 2 * Kp : Kp) * OpTraits<MODE>::kElem;
}

// A operand tiles (hi [then lo] halves along K) straight from the caller's
// antenna-major samples, with the samples' squared norms (the order of the
// training-side packing: real parts, then imaginary parts) and linear terms
// wL <w, x>.  The tile's samples are staged in shared memory (coalesced reads
// along the samples); each thread then writes whole 16-byte K chunks.
template <int MODE>
__global__ void __launch_bounds__(256) batch_gram_pack_a_kernel(const BatchGramJob* __restrict__ jobs, float wL)
{
    using T = OpTraits<MODE>;
    const BatchGramJob& jb = jobs[blockIdx.y];
    const int t = blockIdx.x;
    const int S = jb.S;
    const int s0 = t * kTileM;
    if (s0 >= S) return;
    const int N = jb.N, Kp = jb.Kp, pitch = N + 1;
    const int nr = min(kTileM, S - s0);
    extern __shared__ float2 sx[]; // [kTileM][N + 1]
    for (int idx = threadIdx.x; idx < N * kTileM; idx += blockDim.x) {
        const int k = idx / kTileM, i = idx % kTileM;
        sx[i * pitch + k] = i < nr ? jb.rx[size_t(k) * S + s0 + i] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    uint8_t* tile = jb.a_ops + size_t(t) * tile_bytes<MODE>(kTileM, Kp);
    const int nchunk = Kp / T::kChunk;
    for (int idx = threadIdx.x; idx < kTileM * nchunk; idx += blockDim.x) {
        const int r = idx % kTileM, c = idx / kTileM; // consecutive threads: consecutive rows
        const float2* xr = sx + r * pitch;
        uint32_t hw[4], lw[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) hw[q] = lw[q] = 0u;
#pragma unroll
        for (int e = 0; e < T::kChunk; ++e) {
            const int k = c * T::kChunk + e;
            const float x = k < N ? xr[k].x : (k < 2 * N ? xr[k - N].y : 0.f);
            float hi, lo;
            split_operand<MODE>(x, &hi, &lo);
            if constexpr (T::kTF) {
                hw[e] = __float_as_uint(hi);
                lw[e] = __float_as_uint(lo);
            } else {
                const uint32_t hb = __bfloat16_as_ushort(__float2bfloat16_rn(hi));
                const uint32_t lb = __bfloat16_as_ushort(__float2bfloat16_rn(lo));
                hw[e >> 1] |= hb << (16 * (e & 1));
                lw[e >> 1] |= lb << (16 * (e & 1));
            }
        }
        const size_t off = size_t(c) * (kTileM * 16) + (r >> 3) * 128 + (r & 7) * 16;
        *reinterpret_cast<uint4*>(tile + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        if constexpr (T::kSplit)
            *reinterpret_cast<uint4*>(tile + size_t(nchunk) * (kTileM * 16) + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
    for (int r = threadIdx.x; r < nr; r += blockDim.x) {
        const float2* xr = sx + r * pitch;
        float nv = 0.f;
        for (int k = 0; k < N; ++k) nv = fmaf(xr[k].x, xr[k].x, nv);
        for (int k = 0; k < N; ++k) nv = fmaf(xr[k].y, xr[k].y, nv);
        jb.nrm_s[s0 + r] = nv;
        float l0 = 0.f, l1 = 0.f;
        for (int k = 0; k < N; ++k) {
            const float2 v = xr[k];
            const float w0 = jb.w[k], w1 = jb.w[N + k];
            l0 = fmaf(w0, v.x, fmaf(w1, v.y, l0));
            l1 = fmaf(w0, v.y, fmaf(-w1, v.x, l1));
        }
        jb.lin[s0 + r] = make_float2(wL * l0, wL * l1);
    }
}

// B operand chunks of the job's dictionary (two rows per pair) and per chunk
// the coefficients a*wG and the pair norms.
template <int MODE, int CN>
__global__ void __launch_bounds__(256) batch_gram_pack_b_kernel(const BatchGramJob* __restrict__ jobs, float wG)
{
    using C = Chunk<CN>;
    const BatchGramJob& jb = jobs[blockIdx.y];
    const int c = blockIdx.x;
    if (c >= jb.n_chunks) return;
    const int N = jb.N, Np = jb.Np, Kp = jb.Kp;
    uint8_t* chunk = jb.b_ops + size_t(c) * tile_bytes<MODE>(CN, Kp);
    for (int idx = threadIdx.x; idx < CN * Kp; idx += blockDim.x) {
        const int r = idx / Kp, k = idx % Kp;
        const int b = c * C::kPairs + (r >> 1);
        float x = 0.f;
        if (b < jb.Mp && k < 2 * N) {
            const float2 v = jb.Yd[size_t(b) * Np + (k < N ? k : k - N)];
            // row 2j: [Re y; Im y]; row 2j+1: [-Im y; Re y]
            x = (r & 1) == 0 ? (k < N ? v.x : v.y) : (k < N ? -v.y : v.x);
        }
        float hi, lo;
        split_operand<MODE>(x, &hi, &lo);
        put_operand<MODE>(chunk, CN, r, k, hi);
        if constexpr (OpTraits<MODE>::kSplit) put_operand<MODE>(chunk, CN, r, Kp + k, lo);
    }
    float* bx = jb.bx + size_t(c) * C::kBx;
    for (int i = threadIdx.x; i < C::kFw; i += blockDim.x) {
        float v = 0.f;
        if (i < C::kNrm) {
            const int b = c * C::kPairs + (i >> 1);
            v = b < jb.Mp ? jb.a[2 * b + (i & 1)] * wG : 0.f;
        } else {
            const int b = c * C::kPairs + (i - C::kNrm);
            v = b < jb.Mp ? jb.ew2 * jb.nrm_d[b] : 0.f; // norms pre-scaled by ew log2(e)
        }
        bx[i] = v;
    }
    // fix weights of the pairs and the chunk's gate values (warp 0; 0 in the split forms)
    if (threadIdx.x < 32) {
        float g0 = 0.f, g1 = 0.f;
        for (int p = threadIdx.x; p < C::kPairs; p += 32) {
            const int b = c * C::kPairs + p;
            float fw = 0.f, en = 0.f;
            if (b < jb.Mp) {
                fw = (fabsf(jb.a[2 * b] * wG) + fabsf(jb.a[2 * b + 1] * wG)) * fix_scale<MODE>();
                en = -jb.ew2 * jb.nrm_d[b];
            }
            bx[C::kFw + p] = fw;
            g0 = fmaxf(g0, fw);
            g1 = fmaxf(g1, fw * en);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            g0 = fmaxf(g0, __shfl_xor_sync(0xffffffffu, g0, o));
            g1 = fmaxf(g1, __shfl_xor_sync(0xffffffffu, g1, o));
        }
        if (threadIdx.x < 4) bx[C::kGate + threadIdx.x] = threadIdx.x == 0 ? g0 : (threadIdx.x == 1 ? g1 : 0.f);
    }
}

// 16 pairs (32 accumulator columns) of one sample: kernel values from the Gram
// cross terms, contracted with the pairs' coefficients into the two soft
// outputs.  CHECK: pairs whose error bound exceeds kFixEps are left out and
// returned as bits of the mask (pair j -> bit j).
template <bool CHECK, int CN>
__device__ __forceinline__ uint32_t epilogue_pairs16(const float* gv, const float* xs, int p0, float exn, float m2,
                                                     float& f0, float& f1)
{
    uint32_t mask = 0u;
#pragma unroll
    for (int j = 0; j < 16; j += 2) {
        const int pj = p0 + j; // pair index within the chunk
        const float4 aw = *reinterpret_cast<const float4*>(xs + Chunk<CN>::kAw + 2 * pj); // pairs pj, pj+1
        const float2 nb = *reinterpret_cast<const float2*>(xs + Chunk<CN>::kNrm + pj);
        float2 fw = make_float2(0.f, 0.f);
        if constexpr (CHECK) fw = *reinterpret_cast<const float2*>(xs + Chunk<CN>::kFw + pj);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const float es = exn + (e ? nb.y : nb.x), re = gv[2 * (j + e)], im = gv[2 * (j + e) + 1];
            float kA = ex2(fminf(fmaf(m2, re, es), 0.f));
            float kP = ex2(fminf(fmaf(m2, im, es), 0.f));
            float kM = ex2(fminf(fmaf(-m2, im, es), 0.f));
            if constexpr (CHECK) {
                const float kmax = fmaxf(kA, fmaxf(kP, kM));
                if (kmax * es * (e ? fw.y : fw.x) < -1.f) {
                    mask |= 1u << (j + e);
                    kA = kP = kM = 0.f;
                }
            }
            const float a0 = e ? aw.z : aw.x, a1 = e ? aw.w : aw.y;
            f0 = fmaf(a0, kA, fmaf(a1, kM, f0));
            f1 = fmaf(a0, kP, fmaf(a1, kA, f1));
        }
    }
    return mask;
}

// kAtm (CN = 64): the sample tile's operand lives in tensor memory, copied there once by the
// epilogue warps from the packed tile; the UMMAs read only B from shared memory, and the tile's
// shared memory is free: with 64-column chunks two CTAs share an SM (tensor memory: accumulators
// at columns 0-127, A hi from 128, A lo from 128 + Kp).
template <int MODE, int CN>
__global__ void __launch_bounds__(kThreads, 2)
    batch_gram_kernel(const BatchGramJob* __restrict__ jobs, int n_jobs, const int* __restrict__ tile_prefix, int Kpmax,
                      int stages, int* err, unsigned long long wait_ns)
{
    using T = OpTraits<MODE>;
    using C = Chunk<CN>;
    constexpr bool ATM = C::kAtm;
    // job of this CTA: tile_prefix[j] <= blockIdx.x < tile_prefix[j + 1]
    int lo = 0, hi = n_jobs;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (tile_prefix[mid] <= int(blockIdx.x)) lo = mid;
        else hi = mid;
    }
    const BatchGramJob& jb = jobs[lo];
    const int tile = int(blockIdx.x) - tile_prefix[lo];
    const int nch = jb.n_chunks;

    extern __shared__ __align__(1024) uint8_t smem[];
    const uint32_t a_bytes = uint32_t(tile_bytes<MODE>(kTileM, jb.Kp));
    const uint32_t b_bytes = uint32_t(tile_bytes<MODE>(CN, jb.Kp));
    const uint32_t b_stride = uint32_t(tile_bytes<MODE>(CN, Kpmax));
    uint8_t* sA = smem;
    uint8_t* sB = sA + (ATM ? 0 : tile_bytes<MODE>(kTileM, Kpmax));
    float* sX = reinterpret_cast<float*>(sB + size_t(stages) * b_stride); // [kXRing][C::kBx]
    uint64_t* bars = reinterpret_cast<uint64_t*>(sX + size_t(kXRing) * C::kBx);
    uint64_t* full = bars;                // [stages]
    uint64_t* empty = bars + stages;      // [stages]
    uint64_t* xfull = bars + 2 * stages;  // [kXRing]
    uint64_t* xempty = xfull + kXRing;    // [kXRing]
    uint64_t* tfull = xempty + kXRing;    // [2]
    uint64_t* tempty = tfull + 2;         // [2]
    uint64_t* afull = tempty + 2;         // [1]
    uint64_t* done = afull + 1;           // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    float2* red = reinterpret_cast<float2*>(tmem_slot + 4); // [kTileM]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr uint32_t kCols = ATM ? 4 * CN : 2 * CN; // a power of two: 256
    constexpr uint32_t kAcol = 2 * CN;                // first tensor-memory column of A (ATM)

    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int j = 0; j < kXRing; ++j) {
            mbar_init(&xfull[j], 1);
            mbar_init(&xempty[j], kEpiWarps);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(&tfull[s], 1);
            mbar_init(&tempty[s], kEpiWarps);
        }
        mbar_init(afull, ATM ? kEpiWarps : 1);
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kEpiWarps + 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == kEpiWarps) {
        // ---------------- producer ----------------
        if (lane == 0) {
            if constexpr (!ATM) {
                mbar_expect_tx(afull, a_bytes);
                bulk_g2s(sA, jb.a_ops + size_t(tile) * a_bytes, a_bytes, afull);
            }
            int issued = 0, xissued = 0;
            for (int i = 0; i < nch; ++i) {
                const int s = i % stages, j = i % kXRing;
                if (i >= stages && !mbar_wait(&empty[s], ((i / stages) - 1) & 1, abort_flag, wait_ns)) break;
                ++issued;
                mbar_expect_tx(&full[s], b_bytes);
                bulk_g2s(sB + size_t(s) * b_stride, jb.b_ops + size_t(i) * b_bytes, b_bytes, &full[s]);
                if (i >= kXRing && !mbar_wait(&xempty[j], ((i / kXRing) - 1) & 1, abort_flag, wait_ns)) break;
                ++xissued;
                mbar_expect_tx(&xfull[j], C::kBx * 4);
                bulk_g2s(sX + size_t(j) * C::kBx, jb.bx + size_t(i) * C::kBx, C::kBx * 4, &xfull[j]);
            }
            if constexpr (!ATM) mbar_drain(afull, 0);
            for (int i = max(0, issued - stages); i < issued; ++i) mbar_drain(&full[i % stages], (i / stages) & 1);
            for (int i = max(0, xissued - kXRing); i < xissued; ++i) mbar_drain(&xfull[i % kXRing], (i / kXRing) & 1);
        }
    } else if (warp == kEpiWarps + 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0 && nch > 0 && mbar_wait(afull, 0, abort_flag, wait_ns)) {
            const uint32_t idesc = instr_desc<MODE>(kTileM, CN);
            const uint32_t lbo_a = kTileM * 16, lbo_b = CN * 16;
            const int ksteps = jb.Kp / T::kStepK; // 32 bytes of K per UMMA
            const int lo_off = jb.Kp / T::kChunk; // 16-byte K chunks to the lo half
            for (int i = 0; i < nch; ++i) {
                const int s = i % stages, buf = i & 1;
                if (!mbar_wait(&full[s], (i / stages) & 1, abort_flag, wait_ns)) break;
                if (i >= 2 && !mbar_wait(&tempty[buf], ((i >> 1) - 1) & 1, abort_flag, wait_ns)) break;
                tc_fence_after();
                const uint8_t* b = sB + size_t(s) * b_stride;
                const uint32_t d = tmem + uint32_t(buf * CN);
                for (int kk = 0; kk < ksteps; ++kk) {
                    const uint64_t bh = smem_desc(b + size_t(2 * kk) * lbo_b, lbo_b, 128);
                    if constexpr (ATM) {
                        // A hi / lo of this K step: T::kStepK tensor-memory columns each
                        const uint32_t ah = tmem + kAcol + uint32_t(kk * T::kStepK);
                        const uint64_t bl = smem_desc(b + size_t(lo_off + 2 * kk) * lbo_b, lbo_b, 128);
                        umma_ts<MODE>(d, ah, bh, idesc, kk > 0 ? 1u : 0u);
                        umma_ts<MODE>(d, ah, bl, idesc, 1u);
                        umma_ts<MODE>(d, ah + uint32_t(jb.Kp), bh, idesc, 1u);
                    } else {
                        const uint64_t ah = smem_desc(sA + size_t(2 * kk) * lbo_a, lbo_a, 128);
                        umma<MODE>(d, ah, bh, idesc, kk > 0 ? 1u : 0u);
                        if constexpr (T::kSplit) {
                            const uint64_t al = smem_desc(sA + size_t(lo_off + 2 * kk) * lbo_a, lbo_a, 128);
                            const uint64_t bl = smem_desc(b + size_t(lo_off + 2 * kk) * lbo_b, lbo_b, 128);
                            umma<MODE>(d, ah, bl, idesc, 1u);
                            umma<MODE>(d, al, bh, idesc, 1u);
                        }
                    }
                }
                umma_commit(&tfull[buf]);
                umma_commit(&empty[s]);
            }
        }
        if (lane == 0) {
            umma_commit(done);
            mbar_drain(done, 0);
        }
    } else {
        // ---------------- epilogue ----------------
        const int q = warp & 3, h = warp >> 2;
        if constexpr (ATM) {
            // this warp's 32 rows of the packed sample tile (h = 0: hi half, 1: lo half) into its
            // tensor-memory lanes, 8 columns (two 16-byte K chunks) per store; the MMA waits for all
            const int r = q * 32 + lane;
            const int nck = jb.Kp / T::kChunk;
            const uint8_t* at = jb.a_ops + size_t(tile) * a_bytes + size_t(h * nck) * (kTileM * 16) + (r >> 3) * 128 +
                                (r & 7) * 16;
            const uint32_t tcol = tmem + (uint32_t(q * 32) << 16) + kAcol + uint32_t(h * jb.Kp);
            for (int c = 0; c < nck; c += 2) {
                const uint4 v0 = *reinterpret_cast<const uint4*>(at + size_t(c) * (kTileM * 16));
                const uint4 v1 = *reinterpret_cast<const uint4*>(at + size_t(c + 1) * (kTileM * 16));
                const uint32_t w[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
                tmem_st8(tcol + uint32_t(c * T::kChunk), w);
            }
            tmem_st_wait();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(afull);
        }
        const int row = tile * kTileM + q * 32 + lane;
        const bool valid = row < jb.S;
        const float xn = valid ? jb.nrm_s[row] : 0.f;
        // exponents in base 2: ew log2(e) (|x|^2 + |y|^2 - 2 r) = exn + eyn + m2 r, the pair norms
        // pre-scaled in the chunk data; ew <= 0, so clamping the distance at 0 is clamping the
        // exponent at 0
        const float exn = jb.ew2 * xn, m2 = -2.f * jb.ew2;
        // largest |exn| of the warp's samples (gate of the compensated forms)
        float exn_max = -exn;
        if constexpr (fix_scale<MODE>() > 0.f) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) exn_max = fmaxf(exn_max, __shfl_xor_sync(0xffffffffu, exn_max, o));
        }
        float f0 = 0.f, f1 = 0.f;
        for (int i = 0; i < nch; ++i) {
            const int j = i % kXRing, buf = i & 1;
            if (!mbar_wait(&xfull[j], (i / kXRing) & 1, abort_flag, wait_ns)) break;
            if (!mbar_wait(&tfull[buf], (i >> 1) & 1, abort_flag, wait_ns)) break;
            tc_fence_after();
            const float* xs = sX + size_t(j) * C::kBx;
            // can any pair of this chunk exceed the bound for a sample of this warp?  (warp-uniform)
            const bool check = fix_scale<MODE>() > 0.f && fmaf(exn_max, xs[C::kGate], xs[C::kGate + 1]) > 1.f;
#pragma unroll 1
            for (int cb = 0; cb < CN / 2; cb += 32) {
                const int col = h * (CN / 2) + cb; // 32 columns = 16 pairs
                float gv[32];
                tmem_ld32(tmem + (uint32_t(q * 32) << 16) + uint32_t(buf * CN + col), gv);
                if (!check) {
                    epilogue_pairs16<false, CN>(gv, xs, col >> 1, exn, m2, f0, f1);
                    continue;
                }
                uint32_t mask = epilogue_pairs16<true, CN>(gv, xs, col >> 1, exn, m2, f0, f1);
                if (!valid) mask = 0u;
                // flagged pairs: r = Re(y^H x), m = Im(y^H x) in FP32 from the samples themselves
                while (mask) {
                    const int j = __ffs(mask) - 1;
                    mask &= mask - 1u;
                    const int pj = (col >> 1) + j;
                    const float2* yb = jb.Yd + size_t(i * C::kPairs + pj) * jb.Np;
                    float re = 0.f, im = 0.f;
                    for (int k = 0; k < jb.N; ++k) {
                        const float2 x = jb.rx[size_t(k) * jb.S + row];
                        const float2 y = yb[k];
                        re = fmaf(y.x, x.x, fmaf(y.y, x.y, re));
                        im = fmaf(y.x, x.y, fmaf(-y.y, x.x, im));
                    }
                    const float es = exn + xs[C::kNrm + pj];
                    const float a0 = xs[C::kAw + 2 * pj], a1 = xs[C::kAw + 2 * pj + 1];
                    const float kA = ex2(fminf(fmaf(m2, re, es), 0.f));
                    const float kP = ex2(fminf(fmaf(m2, im, es), 0.f));
                    const float kM = ex2(fminf(fmaf(-m2, im, es), 0.f));
                    f0 = fmaf(a0, kA, fmaf(a1, kM, f0));
                    f1 = fmaf(a0, kP, fmaf(a1, kA, f1));
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&tempty[buf]);
                mbar_arrive(&xempty[j]);
            }
        }
        asm volatile("bar.sync 1, %0;" ::"r"(kEpiWarps * 32) : "memory");
        if (h == 1) red[q * 32 + lane] = make_float2(f0, f1);
        asm volatile("bar.sync 1, %0;" ::"r"(kEpiWarps * 32) : "memory");
        if (h == 0 && row < jb.S) {
            const float2 o = red[q * 32 + lane];
            const float2 l = jb.lin[row];
            jb.out[row] = make_float2(l.x + (f0 + o.x), l.y + (f1 + o.y));
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == kEpiWarps + 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
    }
    if (threadIdx.x == 0 && *abort_flag) atomicExch(err, 1);
}

template <int MODE, int CN> size_t gram_smem(int Kpmax, int stages)
{
    return (Chunk<CN>::kAtm ? 0 : tile_bytes<MODE>(kTileM, Kpmax)) + size_t(stages) * tile_bytes<MODE>(CN, Kpmax) +
           size_t(kXRing) * Chunk<CN>::kBx * 4 + sizeof(uint64_t) * (2 * stages + 2 * kXRing + 6) + 16 +
           sizeof(float2) * kTileM + 1024;
}

template <int MODE, int CN>
cudaError_t launch_cn(const BatchGramJob* d_jobs, int n_jobs, int max_tiles, int max_chunks, const int* d_tile_prefix,
                      int total_tiles, int Kp, float wL, float wG, int* d_err, int stages_req, cudaStream_t s)
{
    // the tile's samples in shared memory: N <= Kp / 2 antennas
    if (max_tiles > 0)
        batch_gram_pack_a_kernel<MODE><<<dim3(max_tiles, n_jobs), 256, sizeof(float2) * kTileM * (Kp / 2 + 1), s>>>(
            d_jobs, wL);
    if (max_chunks > 0) batch_gram_pack_b_kernel<MODE, CN><<<dim3(max_chunks, n_jobs), 256, 0, s>>>(d_jobs, wG);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || total_tiles <= 0) return e;
    // two pipeline stages when that lets two CTAs share an SM, else three if they fit
    // (stages_req 2 or 3 overrides the choice where that many fit)
    constexpr size_t kSmemMax = 227 * 1024;
    int stages = (2 * gram_smem<MODE, CN>(Kp, 3) > kSmemMax) ? 2 : 3;
    if (stages_req == 2 || (stages_req == 3 && gram_smem<MODE, CN>(Kp, 3) <= kSmemMax)) stages = stages_req;
    // every CTA holds 256 TMEM columns: at most two CTAs per SM (512 columns), so
    // shared memory is padded to more than a third of the SM's
    const size_t smem = std::max<size_t>(gram_smem<MODE, CN>(Kp, stages), 80 * 1024);
    e = cudaFuncSetAttribute(batch_gram_kernel<MODE, CN>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    batch_gram_kernel<MODE, CN><<<total_tiles, kThreads, smem, s>>>(d_jobs, n_jobs, d_tile_prefix, Kp, stages, d_err,
                                                                    wait_limit_ns());
    return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_mode(const BatchGramJob* d_jobs, int n_jobs, int max_tiles, int max_chunks,
                        const int* d_tile_prefix, int total_tiles, int Kp, float wL, float wG, int* d_err,
                        int stages_req, cudaStream_t s)
{
    if (Kp % OpTraits<MODE>::kStepK != 0 || Kp > 64) return cudaErrorInvalidValue;
    if constexpr (MODE == kTF32x3) {
        if (chunk_cols(MODE, Kp) == 64)
            return launch_cn<MODE, 64>(d_jobs, n_jobs, max_tiles, max_chunks, d_tile_prefix, total_tiles, Kp, wL, wG,
                                       d_err, stages_req, s);
    }
    return launch_cn<MODE, 128>(d_jobs, n_jobs, max_tiles, max_chunks, d_tile_prefix, total_tiles, Kp, wL, wG, d_err,
                                stages_req, s);
}

} // namespace

int batch_gram_tile() { return kTileM; }
int batch_gram_chunk_pairs(int mode, int Kp) { return chunk_cols(mode, Kp) / 2; }
int batch_gram_kp(int mode, int N)
{
    const int step = (mode == kTF32 || mode == kTF32x3) ? tc::OpTraits<kTF32>::kStepK : tc::OpTraits<kBF16>::kStepK;
    return int(round_up(uint32_t(2 * N), uint32_t(step)));
}
size_t batch_gram_a_bytes(int mode, int Kp)
{
    return size_t(kTileM) * ((mode == kBF16x3 || mode == kTF32x3) ? 2 * Kp : Kp) *
           ((mode == kTF32 || mode == kTF32x3) ? 4 : 2);
}
size_t batch_gram_b_bytes(int mode, int Kp)
{
    return batch_gram_a_bytes(mode, Kp) / kTileM * chunk_cols(mode, Kp);
}
size_t batch_gram_bx_floats(int mode, int Kp) { return 2 * chunk_cols(mode, Kp) + 4; }

cudaError_t launch_batch_gram(int mode, const BatchGramJob* d_jobs, int n_jobs, int max_tiles, int max_chunks,
                              const int* d_tile_prefix, int total_tiles, int Kp, float wL, float wG, int* d_err,
                              int stages, cudaStream_t s)
{
    if (n_jobs <= 0) return cudaSuccess;
    switch (mode) {
    case kBF16:
        return launch_mode<kBF16>(d_jobs, n_jobs, max_tiles, max_chunks, d_tile_prefix, total_tiles, Kp, wL, wG, d_err, stages, s);
    case kBF16x3:
        return launch_mode<kBF16x3>(d_jobs, n_jobs, max_tiles, max_chunks, d_tile_prefix, total_tiles, Kp, wL, wG, d_err,
                                    stages, s);
    case kTF32:
        return launch_mode<kTF32>(d_jobs, n_jobs, max_tiles, max_chunks, d_tile_prefix, total_tiles, Kp, wL, wG, d_err, stages, s);
    case kTF32x3:
        return launch_mode<kTF32x3>(d_jobs, n_jobs, max_tiles, max_chunks, d_tile_prefix, total_tiles, Kp, wL, wG, d_err,
                                    stages, s);
    default:
        return cudaErrorInvalidValue;
    }
}

} // namespace apsm
