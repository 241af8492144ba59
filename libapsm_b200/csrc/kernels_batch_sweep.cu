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
// the reference; results agree to ~1e-6 relative, the FP32 bar is 1e-4):
//   * every window row keeps its whole prediction f_j; after a step it adds
//     sum_i c_i Kt(i, j) with the window kernel Kt = K + wL <x_i, x_j>, which
//     accounts for the change of both a and w;
//   * a pair entering the window starts from wL <x_n, w> + sum_b a_b K(b, n),
//     formed one step ahead from kernel-column values that were prefetched
//     into registers one step before that (rows that already left the window
//     have final coefficients and are read with the prefetch; rows still in
//     the ring come from shared memory);
//   * when the dictionary is full, the evicted pairs' terms leave the sums.
// The window (samples, targets, norms, coefficients, predictions) and its
// kernel, as three planes A / Bp / Bm indexed [row slot][column slot], live in
// shared memory; pair p occupies slot p mod XSP.  Two block barriers per step.
// The kernel has no inter-block waits.
#include "apsm_batch.cuh"

namespace apsm {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kPf = 8;        // prefetched column entries per thread: columns up to kThreads * kPf pairs
constexpr int kParts = 4;     // row-slot parts of the window update
constexpr int kMaxEnter = 4;  // pairs entering per step (sampleStep <= 8)

struct PairStep {
    int hiP, sP, nAP, loP, wk;
};

__device__ __forceinline__ PairStep pair_step(const TrainStep& s, int capP)
{
    PairStep p;
    p.hiP = s.hi >> 1;
    p.sP = (s.hi - s.wk) >> 1;
    p.nAP = s.n_active >> 1;
    p.loP = max(0, p.hiP - capP);
    p.wk = s.wk;
    return p;
}

__device__ __forceinline__ float hyperslab(float e, float eB)
{
    // apsm_train.cu:380-401
    if (e > eB) return __fsub_rn(e, eB);
    if (e < -eB) return __fadd_rn(e, eB);
    return 0.f;
}

// a_{2b} K(2b, .) + a_{2b+1} K(2b+1, .) for the two rows of the column's pair
__device__ __forceinline__ void acc_pair(float2 ab, float4 kv, float& g0, float& g1)
{
    g0 = fmaf(ab.x, kv.x, fmaf(ab.y, kv.z, g0));
    g1 = fmaf(ab.x, kv.y, fmaf(ab.y, kv.x, g1));
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

__global__ void __launch_bounds__(kThreads, 2)
    batch_sweep_kernel(const BatchTrainJob* __restrict__ jobs, int n_jobs, BatchCommon cm, int* counter)
{
    extern __shared__ __align__(16) float smem[];
    __shared__ int job_s;
    const int XSP = cm.XSP, XSPp = cm.XSPp, LB = cm.LB, qP = cm.qP;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const float wL = cm.wL, wG = cm.wG, eB = cm.eB;
    const int Lp = (XSP + kParts - 1) / kParts; // row slots per part
    const int ncp = (XSP + 1) / 2;              // column-slot pairs
    const int halfP = (XSP + 1) / 2;            // row slots per half of the w update

    float* KA = smem;                                        // [XSP][XSPp]
    float* KP = KA + XSP * XSPp;                             // [XSP][XSPp]
    float* KM = KP + XSP * XSPp;                             // [XSP][XSPp]
    float2* Yw = reinterpret_cast<float2*>(KM + XSP * XSPp); // [XSP][Np]
    float* hw = reinterpret_cast<float*>(Yw + XSP * cm.Np);  // [2 XSPp] predictions by row slot
    float* yw = hw + 2 * XSPp;                               // targets
    float* aw = yw + 2 * XSPp;                               // coefficients
    float* cs = aw + 2 * XSPp;                               // corrections of the step (0 when inactive)
    float* nw = cs + 2 * XSPp;                               // [XSPp] norms by pair slot
    float* red = nw + XSPp;                                  // [kParts][2 XSPp] window-update partials
    float* w_s = red + kParts * 2 * XSPp;                    // [kMaxFeatures]
    float* wred = w_s + kMaxFeatures;                        // [2][kMaxFeatures] w-update partials
    float* wp = wred + 2 * kMaxFeatures;                     // [kMaxEnter][kWarps][2] entering partial sums

    for (;;) {
        __syncthreads();
        if (tid == 0) job_s = atomicAdd(counter, 1);
        __syncthreads();
        const int jid = job_s;
        if (jid >= n_jobs) break;
        const BatchTrainJob& jb = jobs[jid];
        const int N = jb.N, Np = jb.Np, capP = jb.capP, nP = jb.nP, n_steps = jb.n_steps;
        const int D = 2 * N;
        const float2* __restrict__ Y = jb.Y;
        float* __restrict__ ag = jb.a;
        const long long kc_base = jb.kc_base;

        auto col_ptr = [&](int n) -> const float4* {
            return jb.Kc + (column_prefix(n, qP, nP, capP) - kc_base) - col_begin(n, capP);
        };
        auto band_ptr = [&](int n) -> const float4* { // indexed by pair b in [n - LB + 1, n]
            return jb.band + size_t(n - jb.n_first) * LB - (n - LB + 1);
        };
        auto slot_of = [&](int p) { return p % XSP; };
        auto pair_in = [&](int q, int lo) { // pair in slot q among the XSP pairs starting at lo
            int d = q - lo % XSP;
            if (d < 0) d += XSP;
            return lo + d;
        };
        auto fill_band = [&](int n, int b, float4 kt) { // window kernel block (b, n) and its transpose
            const int sb = slot_of(b), qn = slot_of(n);
            KA[sb * XSPp + qn] = kt.x;
            KP[sb * XSPp + qn] = kt.y;
            KM[sb * XSPp + qn] = kt.z;
            KA[qn * XSPp + sb] = kt.x;
            KP[qn * XSPp + sb] = kt.z;
            KM[qn * XSPp + sb] = kt.y;
        };
        // linear-term contribution of feature d (< D) of pair value v = y_n[d mod N] with weight wd
        auto lin_feature = [&](int d, float wd, float2 v, float& g0, float& g1) {
            if (d < N) {
                g0 = fmaf(wL * wd, v.x, g0);
                g1 = fmaf(wL * wd, v.y, g1);
            } else {
                g0 = fmaf(wL * wd, v.y, g0);
                g1 = fmaf(-wL * wd, v.x, g1);
            }
        };

        // ---- job state ----
        for (int i = tid; i < 3 * XSP * XSPp; i += kThreads) KA[i] = 0.f;
        for (int i = tid; i < XSP * Np; i += kThreads) Yw[i] = make_float2(0.f, 0.f);
        for (int i = tid; i < 2 * XSPp; i += kThreads) hw[i] = yw[i] = aw[i] = cs[i] = 0.f;
        for (int i = tid; i < XSPp; i += kThreads) nw[i] = 0.f;
        for (int i = tid; i < kParts * 2 * XSPp; i += kThreads) red[i] = 0.f;
        for (int i = tid; i < kMaxFeatures; i += kThreads) {
            w_s[i] = i < D ? jb.w[i] : 0.f;
            wred[i] = wred[kMaxFeatures + i] = 0.f;
        }
        if (n_steps <= 0) continue;
        __syncthreads();

        PairStep pc = pair_step(jb.steps[0], capP);

        // ---- prologue: the pairs of the first window enter with direct loads ----
        {
            const int e_lo = pc.sP, e_hi = pc.hiP, top = jb.used_beforeP;
            for (int j = e_lo + warp; j < e_hi; j += kWarps) {
                const int q = slot_of(j);
                for (int k = lane; k < Np; k += 32) Yw[q * Np + k] = Y[size_t(j) * Np + k];
                float g0 = 0.f, g1 = 0.f;
                const float4* col = col_ptr(j);
                for (int b = pc.loP + lane; b < top; b += 32)
                    acc_pair(*reinterpret_cast<const float2*>(ag + 2 * b), col[b], g0, g1);
                for (int d = lane; d < D; d += 32) lin_feature(d, w_s[d], Y[size_t(j) * Np + d % N], g0, g1);
                warp_sum2(g0, g1);
                if (lane == 0) {
                    hw[2 * q] = g0;
                    hw[2 * q + 1] = g1;
                    yw[2 * q] = jb.y[2 * j];
                    yw[2 * q + 1] = jb.y[2 * j + 1];
                    aw[2 * q] = ag[2 * j];
                    aw[2 * q + 1] = ag[2 * j + 1];
                    nw[q] = jb.nrm[j];
                }
                const float4* bnd = band_ptr(j);
                for (int b = max(e_lo, j - LB + 1) + lane; b <= j; b += 32) fill_band(j, b, bnd[b]);
            }
        }

        // ---- register prefetch for the pair entering at step tt ----
        int pf_n = -1, pf_lo = 0, pf_top = 0, pf_fb = 0;
        float4 pf_k[kPf];
        float2 pf_a[kPf];
        float4 pf_band = make_float4(0.f, 0.f, 0.f, 0.f);
        float2 pf_y = make_float2(0.f, 0.f);
        float pf_t0 = 0.f, pf_t1 = 0.f, pf_nv = 0.f;
        auto prefetch = [&](int tt, int fb) {
            pf_n = -1;
            if (tt <= 0 || tt >= n_steps) return;
            const PairStep ps = pair_step(jb.steps[tt], capP), pv = pair_step(jb.steps[tt - 1], capP);
            const int e_lo = max(pv.hiP, ps.sP);
            if (ps.hiP - e_lo != 1 || pv.hiP - ps.loP > kThreads * kPf || LB > kThreads || D > kThreads)
                return; // direct loads instead
            const int n = e_lo;
            pf_n = n;
            pf_lo = ps.loP;
            pf_top = pv.hiP;
            pf_fb = min(fb, pf_top);
            const float4* col = col_ptr(n);
#pragma unroll
            for (int k = 0; k < kPf; ++k) {
                const int b = pf_lo + tid + k * kThreads;
                pf_k[k] = b < pf_top ? __ldg(col + b) : make_float4(0.f, 0.f, 0.f, 0.f);
                pf_a[k] = b < pf_fb ? *reinterpret_cast<const float2*>(ag + 2 * b) : make_float2(0.f, 0.f);
            }
            if (tid < LB && n - LB + 1 + tid >= 0) pf_band = __ldg(band_ptr(n) + (n - LB + 1 + tid));
            if (tid < D) pf_y = Y[size_t(n) * Np + tid % N];
            if (tid == 0) {
                pf_t0 = jb.y[2 * n];
                pf_t1 = jb.y[2 * n + 1];
                pf_nv = jb.nrm[n];
            }
        };
        prefetch(1, pc.sP);
        __syncthreads();

        TrainStep s_nxt = n_steps > 1 ? jb.steps[1] : jb.steps[0];
#pragma unroll 1
        for (int t = 0; t < n_steps; ++t) {
            const bool has_next = t + 1 < n_steps;
            const PairStep pn = has_next ? pair_step(s_nxt, capP) : pc;
            const int e_lo = has_next ? max(pc.hiP, pn.sP) : 0;
            const int ne = has_next ? max(0, pn.hiP - e_lo) : 0; // pairs entering at t+1

            // ================= phase 1 =================
            // (1a) window rows: fold the last update in; corrections of the active rows
            for (int r = tid; r < 2 * XSP; r += kThreads) {
                const int q = r >> 1;
                const int p = pair_in(q, pc.sP);
                float c = 0.f;
                if (p < pc.hiP) {
                    const float h = hw[r] + ((red[r] + red[2 * XSPp + r]) + (red[4 * XSPp + r] + red[6 * XSPp + r]));
                    hw[r] = h;
                    if (p - pc.sP < pc.nAP) {
                        c = hyperslab(__fsub_rn(yw[r], h), eB);
                        c = __fdiv_rn(c, float(pc.wk));
                        c = __fdiv_rn(c, __fadd_rn(__fmul_rn(wL, nw[q]), wG));
                    }
                }
                cs[r] = c;
            }
            // (1b) w(t): fold the last w update in
            float wd = 0.f;
            if (tid < D) {
                wd = w_s[tid] + (wred[tid] + wred[kMaxFeatures + tid]);
                w_s[tid] = wd;
            }
            // (1c) pairs entering at t+1: data, window kernel, start of their predictions
            if (ne == 1 && pf_n == e_lo) {
                const int n = pf_n, qn = slot_of(n);
                float g0 = 0.f, g1 = 0.f;
#pragma unroll
                for (int k = 0; k < kPf; ++k) {
                    const int b = pf_lo + tid + k * kThreads;
                    if (b < pf_top) {
                        const float2 ab = b < pf_fb ? pf_a[k] : *reinterpret_cast<const float2*>(aw + 2 * slot_of(b));
                        acc_pair(ab, pf_k[k], g0, g1);
                    }
                }
                if (tid < D) lin_feature(tid, wd, pf_y, g0, g1);
                warp_sum2(g0, g1);
                if (lane == 0) {
                    wp[2 * warp] = g0;
                    wp[2 * warp + 1] = g1;
                }
                if (tid < LB && n - LB + 1 + tid >= 0) fill_band(n, n - LB + 1 + tid, pf_band);
                if (tid < Np) Yw[qn * Np + tid] = tid < N ? pf_y : make_float2(0.f, 0.f);
                if (tid == 0) {
                    yw[2 * qn] = pf_t0;
                    yw[2 * qn + 1] = pf_t1;
                    aw[2 * qn] = aw[2 * qn + 1] = 0.f;
                    nw[qn] = pf_nv;
                }
            } else if (ne > 0) {
                // direct loads (several pairs per step, or a column longer than the registers hold)
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
                    if (tid < D) lin_feature(tid, wd, Y[size_t(n) * Np + tid % N], g0, g1);
                    warp_sum2(g0, g1);
                    if (lane == 0) {
                        wp[(e * kWarps + warp) * 2] = g0;
                        wp[(e * kWarps + warp) * 2 + 1] = g1;
                    }
                    const float4* bnd = band_ptr(n);
                    for (int i = tid; i < LB; i += kThreads) {
                        const int b = n - LB + 1 + i;
                        if (b >= 0) fill_band(n, b, bnd[b]);
                    }
                    for (int k = tid; k < Np; k += kThreads) Yw[qn * Np + k] = Y[size_t(n) * Np + k];
                    if (tid == 0) {
                        yw[2 * qn] = jb.y[2 * n];
                        yw[2 * qn + 1] = jb.y[2 * n + 1];
                        aw[2 * qn] = aw[2 * qn + 1] = 0.f;
                        nw[qn] = jb.nrm[n];
                    }
                }
            }
            __syncthreads();

            // ================= phase 2 =================
            // (2a) window update partials and w-update partials
            {
                const int n_h = ncp * kParts, n_w = 2 * D;
                for (int idx = tid; idx < n_h + n_w; idx += kThreads) {
                    if (idx < n_h) {
                        const int cp = idx % ncp, part = idx / ncp;
                        const int p0 = part * Lp, p1 = min(XSP, p0 + Lp);
                        float h00 = 0.f, h01 = 0.f, h10 = 0.f, h11 = 0.f;
                        for (int p = p0; p < p1; ++p) {
                            const float2 c = *reinterpret_cast<const float2*>(cs + 2 * p);
                            const float2 A = *reinterpret_cast<const float2*>(KA + p * XSPp + 2 * cp);
                            const float2 Bp = *reinterpret_cast<const float2*>(KP + p * XSPp + 2 * cp);
                            const float2 Bm = *reinterpret_cast<const float2*>(KM + p * XSPp + 2 * cp);
                            h00 = fmaf(c.x, A.x, fmaf(c.y, Bm.x, h00));
                            h01 = fmaf(c.x, Bp.x, fmaf(c.y, A.x, h01));
                            h10 = fmaf(c.x, A.y, fmaf(c.y, Bm.y, h10));
                            h11 = fmaf(c.x, Bp.y, fmaf(c.y, A.y, h11));
                        }
                        *reinterpret_cast<float4*>(red + part * 2 * XSPp + 4 * cp) = make_float4(h00, h01, h10, h11);
                    } else {
                        const int u = idx - n_h, half = u / D, d = u % D, k = d % N;
                        const int p0 = half * halfP, p1 = min(XSP, p0 + halfP);
                        float acc = 0.f;
                        for (int p = p0; p < p1; ++p) {
                            const float2 c = *reinterpret_cast<const float2*>(cs + 2 * p);
                            const float2 v = Yw[p * Np + k];
                            acc = d < N ? fmaf(c.x, v.x, fmaf(c.y, v.y, acc)) : fmaf(c.x, v.y, fmaf(-c.y, v.x, acc));
                        }
                        wred[half * kMaxFeatures + d] = acc;
                    }
                }
            }
            // (2b) coefficients of the active rows (apsm_train.cu:407)
            for (int r = tid; r < 2 * XSP; r += kThreads) {
                const int p = pair_in(r >> 1, pc.sP);
                if (p < pc.hiP && p - pc.sP < pc.nAP) {
                    const float v = __fadd_rn(aw[r], cs[r]);
                    aw[r] = v;
                    ag[2 * p + (r & 1)] = v;
                }
            }
            // (2c) entering pairs: predictions start from the reduced partial sums
            for (int i = tid; i < 2 * min(ne, kMaxEnter); i += kThreads) {
                const int e = i >> 1, row = i & 1;
                float s = 0.f;
                for (int w2 = 0; w2 < kWarps; ++w2) s += wp[(e * kWarps + w2) * 2 + row];
                hw[2 * slot_of(e_lo + e) + row] = s;
            }
            // (2d) evicted pairs leave the sums of the rows that stay in the window
            if (has_next && pn.loP > pc.loP) {
                for (int r = tid; r < 2 * XSP; r += kThreads) {
                    const int p = pair_in(r >> 1, pn.sP);
                    if (p >= pc.hiP) continue;
                    const float4* col = col_ptr(p);
                    float g0 = 0.f, g1 = 0.f;
                    for (int b = pc.loP; b < pn.loP; ++b)
                        acc_pair(*reinterpret_cast<const float2*>(ag + 2 * b), col[b], g0, g1);
                    hw[r] -= (r & 1) ? g1 : g0;
                }
            }
            // (2e) prefetch for the pair entering at t+2
            prefetch(t + 2, pc.sP);
            if (t + 2 < n_steps) s_nxt = jb.steps[t + 2];
            pc = pn;
            __syncthreads();
        }
        // final linear weights
        if (tid < D) jb.w[tid] = w_s[tid] + (wred[tid] + wred[kMaxFeatures + tid]);
    }
}

int batch_sweep_threads() { return kThreads; }

size_t batch_sweep_smem(const BatchCommon& cm)
{
    const size_t f = 3 * size_t(cm.XSP) * cm.XSPp + 2 * size_t(cm.XSP) * cm.Np + 8 * size_t(cm.XSPp) + cm.XSPp +
                     size_t(kParts) * 2 * cm.XSPp + 3 * kMaxFeatures + 2 * kMaxEnter * kWarps;
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
