// Batched APSM training sweep: one CTA per training job, all jobs in one
// persistent launch (jobs taken in the order given, longest first, from a
// counter).
//
// Model and step semantics are the reference's (cpp/lib/apsm/apsm_train.cu:
// 100-166 host step loop, :271-432 kernel; prediction apsm_detect.cu:170-226):
// at every step each active window row j gets
//     f_j = wL <x_j, w> + sum_{b visible} a_b K(b, j),
//     c_j = hyperslab(y_j - f_j) / W / (wL |x_j|^2 + wG),
// then a_j += c_j and w += sum_j c_j x_j, all from the pre-step values.
//
// Incremental, pair-form evaluation (the floating-point order differs from
// the reference, and the two divisions of the projection are products with
// reciprocals; results agree to ~1e-6 relative, the FP32 bar is 1e-4).  With
// the combined kernel Kt = K + wL <x, x'> and the residual weights
// r = w - sum_{b visible} a_b x_b (zero for a fresh detector),
//     f_j = wL <x_j, r> + sum_{b visible} a_b Kt(b, j),
// and a step changes only window coefficients, so r stays fixed until a
// dictionary entry is evicted (then r += a_b x_b and the entry's K term leaves
// the sums).  Therefore:
//   * every window row keeps its whole prediction; after a step it adds
//     sum_i c_i Kt(i, j) (the window kernel lives in shared memory as three
//     planes A / Bp / Bm indexed [row slot][column slot]; pair p occupies
//     slot p mod XSP);
//   * a pair entering at step t+1 starts from wL <x_n, r> + sum_b a_b Kt(b, n),
//     formed in three stages: its kernel-column values and the coefficients
//     of the pairs that left the window are loaded at step t-2, the part over
//     those final coefficients is summed at step t-1, and the part over the
//     pairs still in the window ring (shared memory) is added at step t;
//   * w = r + sum_b a_b x_b is formed once at the end.
// Two block barriers per step; the kernel has no inter-block waits.
#include "apsm_batch.cuh"

namespace apsm {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kPf = 8;        // frozen column entries per thread: up to kThreads * kPf pairs per column
constexpr int kParts = 6;     // row-slot parts of the window update
constexpr int kMaxEnter = 4;  // pairs entering per step (sampleStep <= 8)
constexpr int kRowThreads = 192;              // warps 0-5: the window rows' corrections
constexpr int kEntThreads = kThreads - kRowThreads; // warps 6-7: the entering pair (window part, linear term)

struct PairStep {
    int hiP, sP, nAP, loP, wk;
};

__device__ __forceinline__ PairStep pair_step(const int4& s, int capP)
{
    // s = TrainStep {hi, wk, n_active, reveal_lo}
    PairStep p;
    p.hiP = s.x >> 1;
    p.sP = (s.x - s.y) >> 1;
    p.nAP = s.z >> 1;
    p.loP = max(0, p.hiP - capP);
    p.wk = s.y;
    return p;
}

// A pair entering the window, as staged by the pipeline: frozen part
// [lo, F) (final coefficients), window part [F, top) (ring coefficients).
struct Entry {
    int n;    // pair, -1 when no pair enters at that step
    int lo, F, top;
    int slow; // served by direct loads when consumed
    int fl;   // first frozen entry staged by this thread block's loads (entries [fl, F))
};

// Bulk prefetch of a global range into L2 (16-byte aligned, size a multiple of 16): a hint, no
// shared memory and no register is involved.
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

constexpr int kPrefetchPairs = 4; // kernel columns brought into L2 this many pairs before their loads

__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float hyperslab(float e, float eB)
{
    // apsm_train.cu:380-401
    if (e > eB) return __fsub_rn(e, eB);
    if (e < -eB) return __fadd_rn(e, eB);
    return 0.f;
}

// a_{2b} Kt(2b, .) + a_{2b+1} Kt(2b+1, .) for the two rows of the column's pair
__device__ __forceinline__ void acc_pair(float2 ab, float4 kv, float& g0, float& g1)
{
    g0 = fmaf(ab.x, kv.x, fmaf(ab.y, kv.z, g0));
    g1 = fmaf(ab.x, kv.y, fmaf(ab.y, kv.x, g1));
}

// asynchronous global -> shared copies (complete at cp_async_wait_all)
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst))),
                 "l"(gmem_src)
                 : "memory");
}

__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst))),
                 "l"(gmem_src)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit_wait_all()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

__device__ __forceinline__ void warp_sum2(float& a, float& b)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
}

} // namespace

#ifdef APSM_SWEEP_PROFILE
// Profiling builds: globaltimer stamps of block 0's jobs (setup, prologue, each step, end).
__device__ unsigned long long g_sweep_prof[64][6]; // start, setup, prologue, steps, final w, n_steps
__device__ unsigned int g_sweep_prof_n;
#define SWEEP_MARK(k)                                                                                        \
    do {                                                                                                     \
        if (blockIdx.x == 0 && tid == 0 && g_sweep_prof_n < 64) {                                           \
            unsigned long long t_;                                                                           \
            asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t_));                                           \
            g_sweep_prof[g_sweep_prof_n][k] = t_;                                                            \
        }                                                                                                    \
    } while (0)
extern "C" void apsm_sweep_prof_read(unsigned long long* out, unsigned int* n)
{
    cudaMemcpyFromSymbol(out, g_sweep_prof, sizeof(g_sweep_prof));
    cudaMemcpyFromSymbol(n, g_sweep_prof_n, sizeof(unsigned int));
    const unsigned int z = 0;
    cudaMemcpyToSymbol(g_sweep_prof_n, &z, sizeof(z));
}
// per-step phase stamps of block 0's first job (clock64): loop top, phase 1 done, window
// update done, evictions done, step end
__device__ long long g_sweep_steps[64][8];
#define STEP_MARK(k)                                                                                         \
    do {                                                                                                     \
        if (blockIdx.x == 0 && tid == 0 && g_sweep_prof_n == 0 && t < 64) g_sweep_steps[t][k] = clock64();  \
    } while (0)
extern "C" void apsm_sweep_steps_read(long long* out)
{
    cudaMemcpyFromSymbol(out, g_sweep_steps, sizeof(g_sweep_steps));
}
#else
#define SWEEP_MARK(k)
#define STEP_MARK(k)
#endif

__global__ void __launch_bounds__(kThreads, 2)
    batch_sweep_kernel(const BatchTrainJob* __restrict__ jobs, int n_jobs, BatchCommon cm, int* counter)
{
    extern __shared__ __align__(16) float smem[];
    __shared__ int job_s;
    __shared__ BatchTrainJob js;
    const int XSP = cm.XSP, XSPp = cm.XSPp, LB = cm.LB, qP = cm.qP;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float wL = cm.wL, wG = cm.wG, eB = cm.eB;
    const int Lp = (XSP + kParts - 1) / kParts; // row slots per part
    const int ncp = (XSP + 1) / 2;              // column-slot pairs
    // n mod XSP without an integer division: q = floor(n M / 2^32) with M = ceil(2^32 / XSP) is
    // floor(n / XSP) for every n < 2^32 / XSP (pair indices are far below); one fixup as a guard
    const uint32_t xsp_magic = uint32_t((0x100000000ull + uint32_t(XSP) - 1) / uint32_t(XSP));
    auto slot_of = [&](int n) {
        int r = n - int(__umulhi(uint32_t(n), xsp_magic)) * XSP;
        return r >= XSP ? r - XSP : r;
    };

    float* KA = smem;                                        // [XSP][XSPp]
    float* KP = KA + XSP * XSPp;                             // [XSP][XSPp]
    float* KM = KP + XSP * XSPp;                             // [XSP][XSPp]
    float2* Yw = reinterpret_cast<float2*>(KM + XSP * XSPp); // [XSP][Np + 1] (odd pitch: row-slot threads
                                                             // reading one feature each hit distinct banks)
    // (the region is rounded up to whole 16-byte units: red below takes float4 stores)
    float* hw = reinterpret_cast<float*>(Yw + round_up(uint32_t(XSP * (cm.Np + 1)), 2u)); // [2 XSPp] predictions
    float* yw = hw + 2 * XSPp;                               // targets
    float* aw = yw + 2 * XSPp;                               // coefficients
    float* cs = aw + 2 * XSPp;                               // corrections of the step (0 when inactive)
    float* rd = cs + 2 * XSPp;                               // [XSPp] 1 / (wL |x|^2 + wG) by pair slot
    float* red = rd + XSPp;                                  // [kParts][2 XSPp] window-update partials
    float* r_s = red + kParts * 2 * XSPp;                    // [kMaxFeatures] residual weights r
    float* dr = r_s + kMaxFeatures;                          // [kMaxFeatures] r increment of an eviction
    float* wp = dr + kMaxFeatures;                           // [kMaxEnter][kWarps][2] entering partial sums (direct loads)
    float* wpf = wp + 2 * kMaxEnter * kWarps;                // [2][kWarps][2] frozen partial sums by step parity
    float* wpe = wpf + 4 * kWarps;                           // [2][2] window part + linear term (warps 6-7)
    float2* ev_y = reinterpret_cast<float2*>(wpe + 4);       // [kMaxEnter][Np] pairs evicted at a step
    float* ev_a = reinterpret_cast<float*>(ev_y + kMaxEnter * cm.Np); // [2 kMaxEnter] their coefficients
    float* wpr = ev_a + 2 * kMaxEnter;                       // [4][2] old-pair sums of entering pairs (slot tt % 4)
    float* nws = wpr + 8;                                    // [XSPp] squared norms by pair slot
    float* ev_n = nws + XSPp;                                // [kMaxEnter] norms of the evicted pairs

    for (;;) {
        __syncthreads();
        if (tid == 0) {
            job_s = atomicAdd(counter, 1);
            if (job_s < n_jobs) js = jobs[job_s];
        }
        __syncthreads();
        if (job_s >= n_jobs) break;
        SWEEP_MARK(0);
        const int N = js.N, Np = js.Np, capP = js.capP, nP = js.nP, n_steps = js.n_steps;
        const int D = 2 * N;
        const float ew = js.ew;
        const float2* __restrict__ Y = js.Y;
        float* __restrict__ ag = js.a;
        const int4* __restrict__ steps = reinterpret_cast<const int4*>(js.steps);

        auto col_ptr = [&](int n) -> const float4* {
            return js.Kc + (column_prefix(n, qP, nP, capP) - js.kc_base) - col_begin(n, capP);
        };
        auto wrap_slot = [&](int s) { return s >= XSP ? s - XSP : (s < 0 ? s + XSP : s); };
        // window kernel block (b, n) and its transpose, slots sb / qn
        auto fill_band = [&](int sb, int qn, float4 kt) {
            KA[sb * XSPp + qn] = kt.x;
            KP[sb * XSPp + qn] = kt.y;
            KM[sb * XSPp + qn] = kt.z;
            KA[qn * XSPp + sb] = kt.x;
            KP[qn * XSPp + sb] = kt.z;
            KM[qn * XSPp + sb] = kt.y;
        };
        // diagonal block of pair n with squared norm nv: r = nv, m = 0 (the Gaussian values as the
        // kernel-column launches form them: 2^(ew log2(e) x) on the SFU)
        auto fill_diag = [&](int qn, float nv) {
            const float b = wG * ex2_approx(ew * 1.4426950408889634f * (2.f * nv));
            KA[qn * XSPp + qn] = fmaf(wL, nv, wG);
            KP[qn * XSPp + qn] = b;
            KM[qn * XSPp + qn] = b;
        };
        // linear-term contribution of feature d (< D) with weight wd of pair value v = y_n[d mod N]
        auto lin_feature = [&](int d, float wd, float2 v, float& g0, float& g1) {
            const float lw = wL * wd;
            if (d < N) {
                g0 = fmaf(lw, v.x, g0);
                g1 = fmaf(lw, v.y, g1);
            } else {
                g0 = fmaf(lw, v.y, g0);
                g1 = fmaf(-lw, v.x, g1);
            }
        };
        // sum_b (a_2b x_2b + a_2b+1 x_2b+1)[d] over pairs [b0, b1) (global state)
        auto ax_sum = [&](int d, int b0, int b1) {
            const int k = d < N ? d : d - N;
            float acc = 0.f;
            for (int b = b0; b < b1; ++b) {
                const float2 ab = *reinterpret_cast<const float2*>(ag + 2 * b);
                const float2 v = Y[size_t(b) * Np + k];
                acc = d < N ? fmaf(ab.x, v.x, fmaf(ab.y, v.y, acc)) : fmaf(ab.x, v.y, fmaf(-ab.y, v.x, acc));
            }
            return acc;
        };

        // ---- job state ----
        for (int i = tid; i < 3 * XSP * XSPp; i += kThreads) KA[i] = 0.f;
        const int YP = Np + 1; // pitch of the window samples
        for (int i = tid; i < XSP * YP; i += kThreads) Yw[i] = make_float2(0.f, 0.f);
        for (int i = tid; i < 2 * XSPp; i += kThreads) hw[i] = yw[i] = aw[i] = cs[i] = 0.f;
        for (int i = tid; i < XSPp; i += kThreads) rd[i] = nws[i] = 0.f;
        for (int i = tid; i < kParts * 2 * XSPp; i += kThreads) red[i] = 0.f;
        PairStep pc = pair_step(n_steps > 0 ? steps[0] : make_int4(0, 0, 0, 0), capP);
        // residual weights as the detector's last sweep left them (0 for a fresh detector), plus the
        // share of the old pairs [0, loP) that leave the dictionary before this call's first step
        for (int d = tid; d < kMaxFeatures; d += kThreads) {
            float r = 0.f;
            if (d < D && !js.fresh) r = js.r[d] + (n_steps > 0 && pc.loP > 0 ? ax_sum(d, 0, pc.loP) : 0.f);
            r_s[d] = r;
        }
        if (n_steps <= 0) continue; // w unchanged
        __syncthreads();

        int4 st_n = steps[n_steps > 1 ? 1 : 0];
        int4 st_nn = steps[n_steps > 2 ? 2 : 0];
        int4 st_3 = steps[n_steps > 3 ? 3 : 0];

        SWEEP_MARK(1);
        // ---- prologue: the pairs of the first window enter with direct loads ----
        {
            const int e_lo = pc.sP, e_hi = pc.hiP, top = js.used_beforeP;
            for (int j = e_lo + warp; j < e_hi; j += kWarps) {
                const int q = j % XSP;
                for (int k = lane; k < Np; k += 32) Yw[q * YP + k] = Y[size_t(j) * Np + k];
                float g0 = 0.f, g1 = 0.f;
                const float4* col = col_ptr(j);
                if (js.pro && j - e_lo < js.pro_w) {
                    // the kernel-column launch summed the old pairs per pass of its column group
                    if (lane == 0) {
                        const int n0 = js.n_first + (j - js.n_first) / kKcolGroup * kKcolGroup;
                        const int nc = min(kKcolGroup, nP - n0);
                        const int b_lo = col_begin(n0, capP), b_hi = col_end(n0 + nc - 1, qP, nP);
                        const float2* pr = js.pro + size_t(j - js.n_first) * js.pro_stride;
                        for (int ps = 0; ps < (b_hi - b_lo + kKcolRows - 1) / kKcolRows; ++ps) {
                            g0 += pr[ps].x;
                            g1 += pr[ps].y;
                        }
                    }
                } else {
#pragma unroll 8
                    for (int b = pc.loP + lane; b < top; b += 32)
                        acc_pair(*reinterpret_cast<const float2*>(ag + 2 * b), __ldg(col + b), g0, g1);
                }
                for (int d = lane; d < D; d += 32) lin_feature(d, r_s[d], Y[size_t(j) * Np + d % N], g0, g1);
                warp_sum2(g0, g1);
                if (lane == 0) {
                    hw[2 * q] = g0;
                    hw[2 * q + 1] = g1;
                    yw[2 * q] = js.y[2 * j];
                    yw[2 * q + 1] = js.y[2 * j + 1];
                    aw[2 * q] = ag[2 * j];
                    aw[2 * q + 1] = ag[2 * j + 1];
                    rd[q] = __frcp_rn(fmaf(wL, js.nrm[j], wG));
                    nws[q] = js.nrm[j];
                }
                for (int b = max(e_lo, j - LB + 1) + lane; b <= j; b += 32) fill_band(b % XSP, q, col[b]);
            }
        }

        // ---- the entering-pair pipeline (see the header) ----
        Entry e_cur{-1, 0, 0, 0, 0, 0}, e_nxt{-1, 0, 0, 0, 0, 0};
        // frozen part of an entering pair's sum: thread tid takes the pairs b = tid + 256 k (mod 2048)
        // of the frozen range; their final coefficients stay in registers (abuf[k] holds a_b of the
        // pair currently in slot k; loaded once, when b first becomes frozen: pairs below cache_F are
        // cached), and only the column entries are loaded for every entering pair
        float4 colbuf[kPf];
        float2 abuf[kPf];
        int cache_F = 0;
        const int et = tid - kRowThreads; // index among the entering warps' threads (< 0: row warps)
        // the pair features d = et and et + kEntThreads of the entering warps' threads (y_n[d mod N])
        const int fk0 = et >= 0 ? et % N : 0, fk1 = et >= 0 ? (et + kEntThreads) % N : 0;
        float4 win_cur0 = make_float4(0.f, 0.f, 0.f, 0.f), win_cur1 = win_cur0, win_nxt0 = win_cur0, win_nxt1 = win_cur0;
        float2 y_cur0 = make_float2(0.f, 0.f), y_cur1 = y_cur0, y_nxt0 = y_cur0, y_nxt1 = y_cur0;
        float t_cur0 = 0.f, t_cur1 = 0.f, n_cur = 0.f, t_nxt0 = 0.f, t_nxt1 = 0.f, n_nxt = 0.f;
        float gf0 = 0.f, gf1 = 0.f; // this thread's part of the frozen sum of e_cur
        // stage 1: loads for the pair entering at step tt (frozen boundary F)
        auto issue = [&](int tt, const int4& st_tt, const int4& st_prev, int F) {
            e_nxt.n = -1;
            e_nxt.slow = 0;
            if (tt <= 0 || tt >= n_steps) return;
            const PairStep ps = pair_step(st_tt, capP), pv = pair_step(st_prev, capP);
            const int e_lo = max(pv.hiP, ps.sP), ne = ps.hiP - e_lo;
            if (ne <= 0) return;
            e_nxt.n = e_lo;
            e_nxt.lo = ps.loP;
            e_nxt.top = pv.hiP;
            e_nxt.F = min(max(F, e_nxt.lo), e_nxt.top);
            // old pairs below n_first were summed by the kernel-column launch (appending calls)
            const int fl = js.pro ? min(max(e_nxt.lo, js.n_first), e_nxt.F) : e_nxt.lo;
            if (ne != 1 || e_nxt.F - fl > kThreads * kPf || e_nxt.top - e_nxt.F > 2 * kEntThreads ||
                D > 2 * kEntThreads) {
                e_nxt.slow = 1;
                return;
            }
            const int n = e_lo;
            const float4* col = col_ptr(n);
            if (tid == 32) {
                // a later pair's column into L2 (it was written long before: in DRAM by now), so that
                // its loads, kPrefetchPairs steps from now, find it there
                const int n2 = n + kPrefetchPairs;
                if (n2 < nP) {
                    const int b0 = col_begin(n2, capP), b1 = col_end(n2, qP, nP);
                    if (b1 > b0) prefetch_l2(col_ptr(n2) + b0, uint32_t(16 * (b1 - b0)));
                }
            }
            if (warp == 5) {
                // the pair's old-pair sums (one per kernel-column pass): lanes take passes, shuffle sum
                float p0 = 0.f, p1 = 0.f;
                if (js.pro) {
                    const int n0 = js.n_first + (n - js.n_first) / kKcolGroup * kKcolGroup;
                    const int nc = min(kKcolGroup, nP - n0);
                    const int b_lo = col_begin(n0, capP), b_hi = col_end(n0 + nc - 1, qP, nP);
                    const float2* pr = js.pro + size_t(n - js.n_first) * js.pro_stride;
                    const int passes = (b_hi - b_lo + kKcolRows - 1) / kKcolRows;
                    for (int ps2 = lane; ps2 < passes; ps2 += 32) {
                        p0 += pr[ps2].x;
                        p1 += pr[ps2].y;
                    }
                }
                warp_sum2(p0, p1);
                if (lane == 0) {
                    wpr[2 * (tt & 3)] = p0;
                    wpr[2 * (tt & 3) + 1] = p1;
                }
            }
            // loads of the later steps: every address clamped into the column / the pair (the entries
            // past its end are masked where they are used), so no instruction here waits for a load
            e_nxt.fl = fl;
            const int fmax = max(fl, e_nxt.F - 1), tmax = max(e_nxt.lo, e_nxt.top - 1);
#pragma unroll
            for (int k = 0; k < kPf; ++k) {
                const int b = fl + ((tid + k * kThreads - fl) & (kThreads * kPf - 1)); // slot k's pair
                colbuf[k] = __ldg(col + min(b, fmax));
                if (b < e_nxt.F && b >= cache_F) abuf[k] = *reinterpret_cast<const float2*>(ag + 2 * b);
            }
            cache_F = max(cache_F, e_nxt.F);
            if (et >= 0) {
                win_nxt0 = __ldg(col + min(e_nxt.F + et, tmax));
                win_nxt1 = __ldg(col + min(e_nxt.F + et + kEntThreads, tmax));
                y_nxt0 = Y[size_t(n) * Np + fk0];
                y_nxt1 = Y[size_t(n) * Np + fk1];
            }
            if (tid == 0) {
                t_nxt0 = js.y[2 * n];
                t_nxt1 = js.y[2 * n + 1];
                n_nxt = js.nrm[n];
            }
        };
        // stage 2: the frozen sum of e_nxt (per-warp partials into wpf[buf]), then e_nxt becomes e_cur
        auto advance = [&](int buf) {
            gf0 = gf1 = 0.f;
            if (e_nxt.n >= 0 && !e_nxt.slow) {
#pragma unroll
                for (int k = 0; k < kPf; ++k) {
                    const int b = e_nxt.fl + ((tid + k * kThreads - e_nxt.fl) & (kThreads * kPf - 1));
                    if (b < e_nxt.F) acc_pair(abuf[k], colbuf[k], gf0, gf1);
                }
                warp_sum2(gf0, gf1);
                if (lane == 0) {
                    wpf[(buf * kWarps + warp) * 2] = gf0;
                    wpf[(buf * kWarps + warp) * 2 + 1] = gf1;
                }
            }
            e_cur = e_nxt;
            win_cur0 = win_nxt0;
            win_cur1 = win_nxt1;
            y_cur0 = y_nxt0;
            y_cur1 = y_nxt1;
            t_cur0 = t_nxt0;
            t_cur1 = t_nxt1;
            n_cur = n_nxt;
        };
        issue(1, st_n, steps[0], pc.sP);
        advance(1);
        issue(2, st_nn, st_n, pc.sP);
        __syncthreads();

        SWEEP_MARK(2);
        int los = pc.sP % XSP; // slot of the window's first pair
#pragma unroll 1
        for (int t = 0; t < n_steps; ++t) {
            const bool has_next = t + 1 < n_steps;
            const PairStep pn = has_next ? pair_step(st_n, capP) : pc;
            const int e_lo = has_next ? max(pc.hiP, pn.sP) : 0;
            const int ne = has_next ? max(0, pn.hiP - e_lo) : 0; // pairs entering at t+1
            const int4 st_4 = t + 4 < n_steps ? steps[t + 4] : st_3;
            const float inv_wk = __frcp_rn(float(pc.wk));

            STEP_MARK(0);
            // ================= phase 1 =================
            const bool fast = ne == 1 && e_cur.n == e_lo && !e_cur.slow;
            // (1a) window rows: fold the last update in; corrections of the active rows
            for (int r = tid; r < 2 * XSP && tid < kRowThreads; r += kRowThreads) {
                const int q = r >> 1;
                int d = q - los;
                if (d < 0) d += XSP;
                float c = 0.f;
                if (d < pc.hiP - pc.sP) {
                    float h = hw[r];
#pragma unroll
                    for (int pt = 0; pt < kParts; ++pt) h += red[pt * 2 * XSPp + r];
                    hw[r] = h;
                    if (d < pc.nAP) c = hyperslab(__fsub_rn(yw[r], h), eB) * inv_wk * rd[q];
                }
                cs[r] = c;
            }
            if (fast && tid == 0) {
                // the entering pair's target, coefficient, projection scale, norm and diagonal block
                // (thread 0 has the slack here; warps 6-7 take the window part below)
                const int qn = slot_of(e_cur.n);
                yw[2 * qn] = t_cur0;
                yw[2 * qn + 1] = t_cur1;
                aw[2 * qn] = aw[2 * qn + 1] = 0.f;
                rd[qn] = __frcp_rn(fmaf(wL, n_cur, wG));
                nws[qn] = n_cur;
                fill_diag(qn, n_cur);
            }
            // (1b) pairs entering at t+1: data, window kernel, start of their predictions
            if (fast) {
              if (et >= 0) {
                const int n = e_cur.n, qn = slot_of(n);
                float g0 = 0.f, g1 = 0.f;
                const int Fs = slot_of(e_cur.F);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int i = et + h * kEntThreads;
                    const int bw = e_cur.F + i;
                    if (bw < e_cur.top) {
                        const float4 kv = h == 0 ? win_cur0 : win_cur1;
                        const int sl = wrap_slot(Fs + i);
                        acc_pair(*reinterpret_cast<const float2*>(aw + 2 * sl), kv, g0, g1);
                        if (bw > n - LB) fill_band(sl, qn, kv);
                    }
                }
                if (et < D) lin_feature(et, r_s[et], y_cur0, g0, g1);
                if (et + kEntThreads < D) lin_feature(et + kEntThreads, r_s[et + kEntThreads], y_cur1, g0, g1);
                warp_sum2(g0, g1);
                if (lane == 0) {
                    wpe[2 * (warp - kRowThreads / 32)] = g0;
                    wpe[2 * (warp - kRowThreads / 32) + 1] = g1;
                }
                if (et < Np) Yw[qn * YP + et] = et < N ? y_cur0 : make_float2(0.f, 0.f);
              }
            } else if (ne > 0) {
                // direct loads (several pairs per step, or columns longer than the pipeline holds)
                const int top = pc.hiP, lo = pn.loP, fb = pc.sP;
                for (int e = 0; e < min(ne, kMaxEnter); ++e) {
                    const int n = e_lo + e, qn = slot_of(n);
                    const float4* col = col_ptr(n);
                    float g0 = 0.f, g1 = 0.f;
                    for (int b = lo + tid; b < top; b += kThreads) {
                        const float2 ab = b < fb ? *reinterpret_cast<const float2*>(ag + 2 * b)
                                                 : *reinterpret_cast<const float2*>(aw + 2 * slot_of(b));
                        acc_pair(ab, col[b], g0, g1);
                    }
                    if (tid < D) lin_feature(tid, r_s[tid], Y[size_t(n) * Np + tid % N], g0, g1);
                    warp_sum2(g0, g1);
                    if (lane == 0) {
                        wp[(e * kWarps + warp) * 2] = g0;
                        wp[(e * kWarps + warp) * 2 + 1] = g1;
                    }
                    for (int b = max(0, n - LB + 1) + tid; b < n; b += kThreads) fill_band(slot_of(b), qn, col[b]);
                    for (int k = tid; k < Np; k += kThreads) Yw[qn * YP + k] = Y[size_t(n) * Np + k];
                    if (tid == 0) {
                        yw[2 * qn] = js.y[2 * n];
                        yw[2 * qn + 1] = js.y[2 * n + 1];
                        aw[2 * qn] = aw[2 * qn + 1] = 0.f;
                        rd[qn] = __frcp_rn(fmaf(wL, js.nrm[n], wG));
                        nws[qn] = js.nrm[n];
                        fill_diag(qn, js.nrm[n]);
                    }
                }
            }
            __syncthreads();
            STEP_MARK(1);

            // ================= phase 2 =================
            // A single pair leaving the dictionary at t+1: its sample, norm and coefficients are
            // fetched now and used after the window update, which hides their load latency.
            const bool evict = has_next && pn.loP > pc.loP;
            const int nev = evict ? pn.loP - pc.loP : 0;
            const bool ev1 = nev == 1;
            const int lons = slot_of(pn.sP);
            if (ev1) { // copied into shared memory in the background
                if (tid < Np) cp_async8(ev_y + tid, Y + size_t(pc.loP) * Np + tid);
                if (tid == Np) cp_async8(ev_a, ag + 2 * pc.loP);
                if (tid == Np + 1) cp_async4(ev_n, js.nrm + pc.loP);
            }
            // (2a) window update partials: red[part][row] = sum_{p in part} c_p Kt(p, .)
            for (int idx = tid; idx < ncp * kParts; idx += kThreads) {
                const int cp = idx % ncp, part = idx / ncp;
                const int p0 = part * Lp, p1 = min(XSP, p0 + Lp);
                float h00 = 0.f, h01 = 0.f, h10 = 0.f, h11 = 0.f;
                const float* pa = KA + 2 * cp;
                const float* pp = KP + 2 * cp;
                const float* pm = KM + 2 * cp;
#pragma unroll 2
                for (int p = p0; p < p1; ++p) {
                    const float2 c = *reinterpret_cast<const float2*>(cs + 2 * p);
                    const float2 A = *reinterpret_cast<const float2*>(pa + p * XSPp);
                    const float2 Bp = *reinterpret_cast<const float2*>(pp + p * XSPp);
                    const float2 Bm = *reinterpret_cast<const float2*>(pm + p * XSPp);
                    h00 = fmaf(c.x, A.x, fmaf(c.y, Bm.x, h00));
                    h01 = fmaf(c.x, Bp.x, fmaf(c.y, A.x, h01));
                    h10 = fmaf(c.x, A.y, fmaf(c.y, Bm.y, h10));
                    h11 = fmaf(c.x, Bp.y, fmaf(c.y, A.y, h11));
                }
                *reinterpret_cast<float4*>(red + part * 2 * XSPp + 4 * cp) = make_float4(h00, h01, h10, h11);
            }
            STEP_MARK(2);
            // (2b) coefficients of the active rows (apsm_train.cu:407)
            for (int r = tid; r < 2 * XSP; r += kThreads) {
                int d = (r >> 1) - los;
                if (d < 0) d += XSP;
                if (d < pc.nAP) {
                    const float v = __fadd_rn(aw[r], cs[r]);
                    aw[r] = v;
                    ag[2 * (pc.sP + d) + (r & 1)] = v;
                }
            }
            // (2c) evicted pairs: dr = sum a_b x_b joins r; their Gaussian terms leave the rows that stay
            if (evict) {
                // the evicted pairs' samples and coefficients, staged once for all window rows
                const bool staged = nev <= kMaxEnter;
                if (ev1) {
                    cp_async_commit_wait_all();
                    STEP_MARK(5);
                    __syncthreads();
                    STEP_MARK(6);
                } else if (staged) {
                    for (int i = tid; i < nev * Np; i += kThreads) ev_y[i] = Y[size_t(pc.loP) * Np + i];
                    for (int i = tid; i < 2 * nev; i += kThreads) ev_a[i] = ag[2 * pc.loP + i];
                    for (int i = tid; i < nev; i += kThreads) ev_n[i] = js.nrm[pc.loP + i];
                    __syncthreads();
                }
                for (int d = tid; d < kMaxFeatures; d += kThreads) {
                    float v = 0.f;
                    if (d < D) {
                        if (staged) {
                            const int k = d < N ? d : d - N;
                            for (int e = 0; e < nev; ++e) {
                                const float2 ab = make_float2(ev_a[2 * e], ev_a[2 * e + 1]);
                                const float2 yv = ev_y[e * Np + k];
                                v = d < N ? fmaf(ab.x, yv.x, fmaf(ab.y, yv.y, v)) : fmaf(ab.x, yv.y, fmaf(-ab.y, yv.x, v));
                            }
                        } else {
                            v = ax_sum(d, pc.loP, pn.loP);
                        }
                    }
                    dr[d] = v;
                    r_s[d] += v;
                }
                for (int q = tid; q < XSP; q += kThreads) {
                    int dd = q - lons;
                    if (dd < 0) dd += XSP;
                    const int p = pn.sP + dd;
                    if (p >= pc.hiP) continue;
                    float g0 = 0.f, g1 = 0.f;
                    // the Gaussian kernel of pair b against the row's pair, from y_b^H y_p and the norms
                    // (the expressions of the kernel columns)
                    auto evict_term = [&](const float2* yrow, float nb, float2 ab) {
                        float re = 0.f, im = 0.f;
#pragma unroll 4
                        for (int k = 0; k < N; ++k) {
                            const float2 yb = yrow[k], yj = Yw[q * YP + k];
                            re = fmaf(yb.x, yj.x, fmaf(yb.y, yj.y, re));
                            im = fmaf(yb.x, yj.y, fmaf(-yb.y, yj.x, im));
                        }
                        const float sn = nb + nws[q];
                        const float4 kg = make_float4(wG * expf(ew * fmaxf(fmaf(-2.f, re, sn), 0.f)),
                                                      wG * expf(ew * fmaxf(fmaf(-2.f, im, sn), 0.f)),
                                                      wG * expf(ew * fmaxf(fmaf(2.f, im, sn), 0.f)), 0.f);
                        acc_pair(ab, kg, g0, g1);
                    };
                    if (staged) {
                        for (int e = 0; e < nev; ++e)
                            evict_term(ev_y + e * Np, ev_n[e], make_float2(ev_a[2 * e], ev_a[2 * e + 1]));
                    } else {
                        for (int b = pc.loP; b < pn.loP; ++b)
                            evict_term(Y + size_t(b) * Np, js.nrm[b], *reinterpret_cast<const float2*>(ag + 2 * b));
                    }
                    hw[2 * q] -= g0;
                    hw[2 * q + 1] -= g1;
                }
                STEP_MARK(7);
                __syncthreads();
            }
            STEP_MARK(3);
            // (2d) entering pairs: predictions start from the reduced partial sums (plus wL <x_n, dr>
            //      after an eviction: their partial sums used r from before it)
            for (int i = kThreads - 1 - tid; i < 2 * min(ne, kMaxEnter) && i >= 0; i += kThreads) {
                const int e = i >> 1, row = i & 1, qn = slot_of(e_lo + e);
                float s = 0.f;
                if (fast) {
                    const int fb = (t + 1) & 1; // frozen partials of the pair entering at t+1
                    for (int w2 = 0; w2 < kWarps; ++w2) s += wpf[(fb * kWarps + w2) * 2 + row];
                    s += wpr[2 * ((t + 1) & 3) + row];
                    s += wpe[row] + wpe[2 + row];
                } else {
                    for (int w2 = 0; w2 < kWarps; ++w2) s += wp[(e * kWarps + w2) * 2 + row];
                }
                if (evict) {
                    float l = 0.f;
                    for (int k = 0; k < N; ++k) {
                        const float2 v = Yw[qn * YP + k];
                        l = row == 0 ? fmaf(dr[k], v.x, fmaf(dr[N + k], v.y, l)) : fmaf(dr[k], v.y, fmaf(-dr[N + k], v.x, l));
                    }
                    s = fmaf(wL, l, s);
                }
                hw[2 * qn + row] = s;
            }
            STEP_MARK(4);
            // (2e) pipeline: frozen part of the pair entering at t+2, loads for t+3
            advance(t & 1); // the pair entering at t+2: parity (t + 2) & 1
            issue(t + 3, st_3, st_nn, pc.sP);
            los += pn.sP - pc.sP;
            if (los >= XSP) los -= XSP;
            pc = pn;
            st_n = st_nn;
            st_nn = st_3;
            st_3 = st_4;
            __syncthreads();
        }
        SWEEP_MARK(3);
        // w = r + sum over the visible pairs of a_b x_b: warp w2 sums pairs lo + w2 + 8 i, lane k
        // features k and N + k; the warps' sums are added in warp order (the window kernel's
        // shared memory is free now).  r stays with the detector for its next sweep.
        {
            float* part = KA; // [kWarps][kMaxFeatures]
            for (int k = lane; k < kMaxFeatures / 2; k += 32) {
                float s0 = 0.f, s1 = 0.f;
                if (k < N) {
#pragma unroll 4
                    for (int b = pc.loP + warp; b < pc.hiP; b += kWarps) {
                        const float2 ab = *reinterpret_cast<const float2*>(ag + 2 * b);
                        const float2 v = Y[size_t(b) * Np + k];
                        s0 = fmaf(ab.x, v.x, fmaf(ab.y, v.y, s0));
                        s1 = fmaf(ab.x, v.y, fmaf(-ab.y, v.x, s1));
                    }
                }
                part[warp * kMaxFeatures + k] = s0;
                part[warp * kMaxFeatures + kMaxFeatures / 2 + k] = s1;
            }
            __syncthreads();
            for (int d = tid; d < D; d += kThreads) {
                const int idx = d < N ? d : kMaxFeatures / 2 + (d - N);
                float acc = 0.f;
                for (int w2 = 0; w2 < kWarps; ++w2) acc += part[w2 * kMaxFeatures + idx];
                js.w[d] = r_s[d] + acc;
                js.r[d] = r_s[d];
            }
        }
#ifdef APSM_SWEEP_PROFILE
        __syncthreads();
        if (blockIdx.x == 0 && tid == 0 && g_sweep_prof_n < 64) {
            unsigned long long t_;
            asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t_));
            g_sweep_prof[g_sweep_prof_n][4] = t_;
            g_sweep_prof[g_sweep_prof_n][5] = (unsigned long long)n_steps;
            ++g_sweep_prof_n;
        }
#endif
    }
}

int batch_sweep_threads() { return kThreads; }

size_t batch_sweep_smem(const BatchCommon& cm)
{
    const size_t f = 3 * size_t(cm.XSP) * cm.XSPp + 2 * size_t(round_up(uint32_t(cm.XSP * (cm.Np + 1)), 2u)) +
                     8 * size_t(cm.XSPp) + cm.XSPp +
                     size_t(kParts) * 2 * cm.XSPp + 2 * kMaxFeatures + 2 * kMaxEnter * kWarps + 4 * kWarps + 4 +
                     2 * size_t(kMaxEnter) * cm.Np + 2 * kMaxEnter + 8 + cm.XSPp + kMaxEnter;
    return sizeof(float) * f;
}

cudaError_t batch_sweep_occupancy(const BatchCommon& cm, int* ctas_per_sm)
{
    const size_t smem = batch_sweep_smem(cm);
    cudaError_t e = cudaFuncSetAttribute(batch_sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, batch_sweep_kernel, kThreads, smem);
}

cudaError_t launch_batch_sweep(const BatchTrainJob* d_jobs, int n_jobs, BatchCommon cm, int grid, int* d_counter,
                               int* d_err, cudaStream_t s)
{
    (void)d_err;
    if (n_jobs <= 0) return cudaSuccess;
    const size_t smem = batch_sweep_smem(cm);
    cudaError_t e = cudaFuncSetAttribute(batch_sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    batch_sweep_kernel<<<grid, kThreads, smem, s>>>(d_jobs, n_jobs, cm, d_counter);
    return cudaGetLastError();
}

} // namespace apsm
