// APSM training sweep, incremental form (config "trainVersion": "incremental").
//
// Same model and step semantics as the exact sweep (kernels_sweep.cu;
// reference cpp/lib/apsm/apsm_train.cu:100-166, :271-432), but the Gaussian
// part of each window row's prediction
//     g_j = sum_{b visible} a_b K(b, j)
// is kept up to date instead of being re-summed every step: when row j
// enters the window its sum is formed once (from K values prefetched into
// registers during the step before), and after every step each window row
// adds the step's corrections, g_j += sum_{i active} c_i K(i, j).  Per step
// that is W x W multiply-adds instead of W x M; f_j = wL <x_j, w> + g_j.  The
// floating-point order differs from the reference's per-lane order; results
// agree to ~1e-6 relative (the FP32 bar is 1e-4).
//
// A cluster of C CTAs per user (C = 1 allowed).  Window row v is owned by CTA
// v % C, which keeps its Gaussian sum and its column of the window's kernel
// block, Kwin[row slot][owned slot].  Rows live in row slot r % XS and owned
// columns in owned slot (v / C) % NSO.  The window rows, coefficients and
// linear weights are replicated.  A step's corrections are pushed to every
// CTA with st.async; each CTA's mbarrier completes when all of them landed.
// Everything a step needs from HBM/L2 is loaded into registers one step
// ahead.  Waits are bounded (2 s); on expiry args.err is set.
#include "apsm_kernels.cuh"

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace apsm {

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kRowsPerThread = 8; // full sums of entering columns from registers: M <= kThreads * kRowsPerThread
constexpr int kMaxEnter = 4;      // entering rows per step served from registers (more: direct loads)
constexpr int kFillA = 4;         // per-thread fill values: entering rows x owned columns
constexpr int kFillB = 4;         // per-thread fill values: owned entering columns x row slots
constexpr int kParts = 4;         // threads per owned column in the correction update
constexpr int kRowLanes = 8;      // lanes per row in the prediction dot product

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        for (int i = 0; i < 256; ++i)
            if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > 2000000000ull) return false;
    }
}

__device__ __forceinline__ void st_async_f32(const float* local, const uint64_t* bar, uint32_t rank, float v)
{
    uint32_t raddr, rbar;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(raddr) : "r"(smem_u32(local)), "r"(rank));
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(rbar) : "r"(smem_u32(bar)), "r"(rank));
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];" ::"r"(raddr),
                 "r"(__float_as_uint(v)), "r"(rbar)
                 : "memory");
}

// K(u, v) read from column v (rows [column_base(v), v + q2)); 0 outside.
__device__ __forceinline__ float kval(const TrainArgs& a, int u, int v)
{
    const int ub = column_base(v, a.cap);
    if (u < ub || u >= v + a.q2 || u >= a.nU || v < a.v_first || u < 0) return 0.f;
    return __ldg(a.K + size_t(v - a.v_first) * a.Lk + (u - ub));
}

__device__ __forceinline__ int wrap(int s, int n) { return s >= n ? s - n : s; }

} // namespace

// Shared memory (floats unless noted):
//   Kwin  [XS][NSOp]  kernel values K(row of slot si, owned column of slot so)
//   xw    [XS][XP]    window rows (replicated), yw/nw [XS] targets / norms
//   cs    [2][XS]     corrections of the step by row slot (st.async target), 0 elsewhere
//   gown  [NSOp]      Gaussian sums of the owned columns
//   red   [kParts][NSOp]
//   a_ring[A_ring], w_s[128], wpart[kMaxEnter][kWarps]
//   rowof [XS] (int), colof [NSOp] (int), 2 mbarriers, abort flag
__global__ void __launch_bounds__(kThreads, 1) train_inc_kernel(TrainArgs args)
{
    cg::cluster_group cluster = cg::this_cluster();
    const int C = int(cluster.num_blocks());
    const int rank = int(cluster.block_rank());
    const int user = blockIdx.x / C;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int D = args.D, Dp = args.Dp, XP = args.XP, cap = args.cap;
    const int XS = args.XS, NSO = args.NSO, NSOp = args.NSOp; // owned slots and their padded pitch
    const int amask = args.A_ring - 1;
    const int n_steps = args.n_steps;
    const ModelParams mp = args.mp;

    extern __shared__ __align__(16) float smem[];
    float* Kwin = smem;                          // [XS][NSOp]
    float* xw = Kwin + size_t(XS) * NSOp;        // [XS][XP]
    float* yw = xw + size_t(XS) * XP;            // [XS]
    float* nw = yw + XS;                         // [XS]
    float* cs2 = nw + XS;                        // [2][XS]
    float* gown = cs2 + 2 * XS;                  // [NSOp]
    float* red = gown + NSOp;                    // [kParts][NSOp]
    float* a_ring = red + kParts * NSOp;         // [A_ring]
    float* w_s = a_ring + args.A_ring;           // [128]
    float* wpart = w_s + kMaxFeatures;           // [kMaxEnter][kWarps]
    int* rowof = reinterpret_cast<int*>(wpart + kMaxEnter * kWarps); // [XS]
    int* colof = rowof + XS;                                          // [NSOp]
    uint64_t* cfull = reinterpret_cast<uint64_t*>(colof + NSOp + ((XS + NSOp) & 1)); // [2], 8-byte aligned
    volatile int* abort_flag = reinterpret_cast<volatile int*>(cfull + 2);

    const float* __restrict__ X = args.X;
    const float* __restrict__ nrm = args.nrm;
    const float* __restrict__ y = args.y + size_t(user) * args.y_stride;
    float* __restrict__ a_out = args.a + size_t(user) * args.a_stride;
    float* __restrict__ w_out = args.w + size_t(user) * D;

    auto load_step = [&](int tt) -> TrainStep { return (tt >= 0 && tt < n_steps) ? args.steps[tt] : TrainStep{0, 0, 0, 0}; };
    auto enter_lo = [&](int tt, const TrainStep& s, const TrainStep& prev) -> int {
        const int st = s.hi - s.wk;
        return tt == 0 ? st : max(st, prev.hi);
    };
    auto owned = [&](int v) { return v % C == rank; };
    auto oslot = [&](int v) { return (v / C) % NSO; };

    // ---- initial state ----
    for (int i = tid; i < XS * NSOp; i += kThreads) Kwin[i] = 0.f;
    for (int i = tid; i < XS * XP; i += kThreads) xw[i] = 0.f;
    for (int i = tid; i < XS; i += kThreads) {
        yw[i] = nw[i] = cs2[i] = cs2[XS + i] = 0.f;
        rowof[i] = -1;
    }
    for (int i = tid; i < NSOp; i += kThreads) {
        gown[i] = 0.f;
        colof[i] = -1;
    }
    for (int u = tid; u < args.used_before; u += kThreads) a_ring[u & amask] = a_out[u];
    for (int d = tid; d < kMaxFeatures; d += kThreads) w_s[d] = d < D ? w_out[d] : 0.f;
    if (tid == 0) {
        mbar_init(&cfull[0], 1);
        mbar_init(&cfull[1], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // Rows [r0, r1) become resident; owned ones get Gaussian sums over rows
    // [lo, top) with the current coefficients.  Direct global loads
    // (prologue and steps whose entering rows exceed the registers).
    auto enter_direct = [&](int r0, int r1, int lo, int top) {
        for (int r = r0 + warp; r < r1; r += kWarps) {
            const int sl = r % XS;
            for (int d = lane; d < Dp; d += 32) xw[sl * XP + d] = X[size_t(r) * Dp + d];
            if (lane == 0) {
                yw[sl] = y[r];
                nw[sl] = nrm[r];
                rowof[sl] = r;
            }
            if (owned(r)) {
                float p = 0.f;
                for (int b = lo + lane; b < top; b += 32) p = fmaf(a_ring[b & amask], kval(args, b, r), p);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
                if (lane == 0) {
                    gown[oslot(r)] = p;
                    colof[oslot(r)] = r;
                }
            }
        }
        __syncthreads();
        // Kwin: entering rows against owned columns, owned entering columns against all rows
        for (int idx = tid; idx < (r1 - r0) * NSO; idx += kThreads) {
            const int r = r0 + idx / NSO, so = idx % NSO;
            const int col = colof[so];
            Kwin[(r % XS) * NSOp + so] = col >= 0 ? kval(args, r, col) : 0.f;
        }
        for (int idx = tid; idx < (r1 - r0) * XS; idx += kThreads) {
            const int r = r0 + idx / XS, si = idx % XS;
            if (!owned(r)) continue;
            const int row = rowof[si];
            Kwin[si * NSOp + oslot(r)] = row >= 0 ? kval(args, row, r) : 0.f;
        }
        __syncthreads();
    };

    // ---- register prefetch for the rows entering at step tt ----
    int pf_n = 0, pf_e0 = 0, pf_lo = 0, pf_top = 0;
    float pf_kf[kMaxEnter][kRowsPerThread];
    float pf_fa[kFillA], pf_fb[kFillB];
    float pf_x[2], pf_y = 0.f, pf_nv = 0.f;
    auto prefetch = [&](int tt, const TrainStep& s, const TrainStep& prev) {
        pf_n = 0;
        if (tt <= 0 || tt >= n_steps) return;
        pf_e0 = enter_lo(tt, s, prev);
        const int ne = s.hi - pf_e0;
        pf_lo = max(0, s.hi - cap); // visible at tt and at tt-1 (rows revealed at tt have a = 0)
        pf_top = prev.hi;
        if (ne <= 0) return;
        if (ne > kMaxEnter || pf_top - pf_lo > kThreads * kRowsPerThread || ne * NSO > kThreads * kFillA ||
            ne * XS > kThreads * kFillB || ne * Dp > 2 * kThreads) {
            pf_n = -1;
            return;
        }
        pf_n = ne;
        // full sums of the owned entering columns
#pragma unroll
        for (int e = 0; e < kMaxEnter; ++e) {
            const int v = pf_e0 + e;
            const bool use = e < ne && owned(v);
            const int ub = column_base(v, cap);
            const float* col = args.K + size_t(max(0, v - args.v_first)) * args.Lk - ub;
#pragma unroll
            for (int k = 0; k < kRowsPerThread; ++k) {
                const int b = pf_lo + tid + k * kThreads;
                pf_kf[e][k] = (use && b < pf_top) ? __ldg(col + b) : 0.f;
            }
        }
        // Kwin fill (a): entering row r against the owned column of slot so,
        // as it will be after this step's entries (owned entering columns included)
#pragma unroll
        for (int k = 0; k < kFillA; ++k) {
            const int idx = tid + k * kThreads;
            float v = 0.f;
            if (idx < ne * NSO) {
                const int r = pf_e0 + idx / NSO, so = idx % NSO;
                int col = colof[so];
                for (int e2 = 0; e2 < ne; ++e2)
                    if (owned(pf_e0 + e2) && oslot(pf_e0 + e2) == so) col = pf_e0 + e2;
                v = col >= 0 ? kval(args, r, col) : 0.f;
            }
            pf_fa[k] = v;
        }
        // Kwin fill (b): owned entering column r against the row of slot si
#pragma unroll
        for (int k = 0; k < kFillB; ++k) {
            const int idx = tid + k * kThreads;
            float v = 0.f;
            if (idx < ne * XS) {
                const int r = pf_e0 + idx / XS, si = idx % XS;
                if (owned(r)) {
                    int row = rowof[si];
                    for (int e2 = 0; e2 < ne; ++e2)
                        if ((pf_e0 + e2) % XS == si) row = pf_e0 + e2;
                    v = row >= 0 ? kval(args, row, r) : 0.f;
                }
            }
            pf_fb[k] = v;
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int idx = tid + k * kThreads;
            pf_x[k] = idx < ne * Dp ? X[size_t(pf_e0 + idx / Dp) * Dp + idx % Dp] : 0.f;
        }
        pf_y = tid < ne ? y[pf_e0 + tid] : 0.f;
        pf_nv = tid < ne ? nrm[pf_e0 + tid] : 0.f;
    };

    TrainStep s_cur = load_step(0), s_nxt = load_step(1), s_nn = load_step(2);
    if (n_steps > 0) {
        for (int u = s_cur.reveal_lo + tid; u < s_cur.hi; u += kThreads) a_ring[u & amask] = 0.f;
        __syncthreads();
        enter_direct(s_cur.hi - s_cur.wk, s_cur.hi, max(0, s_cur.hi - cap), s_cur.hi);
        if (tid == 0) mbar_expect_tx(&cfull[0], uint32_t(s_cur.n_active) * 4u);
    }
    prefetch(1, s_nxt, s_cur);
    cluster.sync(); // every CTA resident and its barriers armed before the first st.async

#pragma unroll 1
    for (int t = 0; t < n_steps; ++t) {
        const TrainStep st = s_cur;
        const int start = st.hi - st.wk;
        const int s0 = start % XS; // slot of the first window row
        const bool has_next = t + 1 < n_steps;
        float* cs = cs2 + (t & 1) * XS;
        uint64_t* bar = &cfull[t & 1];

        // ---------------- phase A ----------------
        if (pf_n > 0) {
            // (A1) rows entering at t+1: resident data; full-sum partials of owned ones with a(t)
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int idx = tid + k * kThreads;
                if (idx < pf_n * Dp) xw[((pf_e0 + idx / Dp) % XS) * XP + idx % Dp] = pf_x[k];
            }
            if (tid < pf_n) {
                const int sl = (pf_e0 + tid) % XS;
                yw[sl] = pf_y;
                nw[sl] = pf_nv;
            }
#pragma unroll
            for (int e = 0; e < kMaxEnter; ++e) {
                if (e >= pf_n) break;
                if (!owned(pf_e0 + e)) continue;
                float p = 0.f;
#pragma unroll
                for (int k = 0; k < kRowsPerThread; ++k) {
                    const int b = pf_lo + tid + k * kThreads;
                    if (b < pf_top) p = fmaf(a_ring[b & amask], pf_kf[e][k], p);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
                if (lane == 0) wpart[e * kWarps + warp] = p;
            }
        }
        // (A2) predictions and projections of the owned active rows, 8 lanes per row
        {
            const int first = start + ((rank - start % C) + C) % C;
            const int n_own = first < start + st.n_active ? (start + st.n_active - 1 - first) / C + 1 : 0;
            constexpr int kGroups = kThreads / kRowLanes;
            const int grp = tid / kRowLanes, gl = tid % kRowLanes;
            const int rounds = (n_own + kGroups - 1) / kGroups; // uniform across the block (shuffles below)
            for (int rnd = 0; rnd < rounds; ++rnd) {
                const int k = rnd * kGroups + grp;
                const bool valid = k < n_own;
                const int v = first + k * C;
                const int sl = valid ? v % XS : 0;
                float lin = 0.f;
                if (valid)
                    for (int d = gl; d < D; d += kRowLanes) lin = fmaf(xw[sl * XP + d], w_s[d], lin);
#pragma unroll
                for (int o = kRowLanes / 2; o > 0; o >>= 1) lin += __shfl_xor_sync(0xffffffffu, lin, o);
                float c = 0.f;
                if (valid && gl == 0) {
                    const float f = fmaf(mp.wL, lin, gown[oslot(v)]);
                    // hyperslab projection (apsm_train.cu:380-401)
                    const float e = __fsub_rn(yw[sl], f);
                    if (e > mp.eB) c = __fsub_rn(e, mp.eB);
                    else if (e < -mp.eB) c = __fadd_rn(e, mp.eB);
                    const float linearNorm = __fmul_rn(mp.wL, nw[sl]);
                    c = __fdiv_rn(c, float(st.wk));
                    c = __fdiv_rn(c, __fadd_rn(linearNorm, mp.wG));
                }
                c = __shfl_sync(0xffffffffu, c, (lane / kRowLanes) * kRowLanes);
                if (valid)
                    for (int r = gl; r < C; r += kRowLanes) st_async_f32(cs + sl, bar, uint32_t(r), c);
            }
        }
        if (pf_n > 0 && tid < pf_n) {
            const int r = pf_e0 + tid;
            rowof[r % XS] = r;
            if (owned(r)) colof[oslot(r)] = r;
        }
        // next step's barrier can be armed now (its previous phase completed at step t-1)
        if (tid == 0 && has_next) mbar_expect_tx(&cfull[(t + 1) & 1], uint32_t(s_nxt.n_active) * 4u);
        if (!mbar_wait_bounded(bar, uint32_t(t >> 1) & 1u)) *abort_flag = 1;
        __syncthreads();
        if (*abort_flag) break;

        // ---------------- phase B ----------------
        // (B0) Kwin entries of the rows / owned columns entering at t+1
        if (pf_n > 0) {
#pragma unroll
            for (int k = 0; k < kFillA; ++k) {
                const int idx = tid + k * kThreads;
                if (idx < pf_n * NSO) Kwin[((pf_e0 + idx / NSO) % XS) * NSOp + idx % NSO] = pf_fa[k];
            }
#pragma unroll
            for (int k = 0; k < kFillB; ++k) {
                const int idx = tid + k * kThreads;
                if (idx < pf_n * XS) {
                    const int r = pf_e0 + idx / XS;
                    if (owned(r)) Kwin[(idx % XS) * NSOp + oslot(r)] = pf_fb[k];
                }
            }
        }
        // (B1) a_j += c_j (apsm_train.cu:407)
        for (int i = tid; i < st.n_active; i += kThreads) {
            float* ap = a_ring + ((start + i) & amask);
            *ap = __fadd_rn(*ap, cs[wrap(s0 + i, XS)]);
        }
        // (B2) w += sum_j c_j x_j (apsm_train.cu:413-428)
        {
            const int nwork = int(round_up(uint32_t(D * kWGroups), 32u));
            for (int idx = tid; idx < nwork; idx += kThreads) {
                const int d = idx / kWGroups, gi = idx % kWGroups;
                float acc = 0.f;
                if (d < D) {
                    int sl = wrap(s0 + gi, XS);
                    for (int i = gi; i < st.n_active; i += kWGroups) {
                        acc = fmaf(cs[sl], xw[sl * XP + d], acc);
                        sl = wrap(sl + kWGroups, XS);
                    }
                }
                acc += __shfl_xor_sync(0xffffffffu, acc, 1);
                acc += __shfl_xor_sync(0xffffffffu, acc, 2);
                acc += __shfl_xor_sync(0xffffffffu, acc, 4);
                if (d < D && gi == 0) w_s[d] += acc;
            }
        }
        __syncthreads(); // Kwin entries complete
        if (args.snap_a && rank == 0) {
            // training history: the model after this step (a_j and w are final here and not
            // written again before the next step's barriers)
            float* sa = args.snap_a + (size_t(user) * n_steps + t) * args.q2;
            for (int i = tid; i < st.n_active; i += kThreads) sa[i] = a_ring[(start + i) & amask];
            float* sw = args.snap_w + (size_t(user) * n_steps + t) * D;
            for (int d = tid; d < D; d += kThreads) sw[d] = w_s[d];
        }
        // (B3) owned column sums: g += sum_si cs[si] Kwin[si][so]
        for (int idx = tid; idx < kParts * NSOp; idx += kThreads) {
            const int part = idx / NSOp, so = idx % NSOp;
            float acc = 0.f;
            if (so < NSO)
                for (int si = part; si < XS; si += kParts) acc = fmaf(cs[si], Kwin[si * NSOp + so], acc);
            red[part * NSOp + so] = acc;
        }
        // rows revealed at t+1 start with a = 0 (not visible now)
        if (has_next)
            for (int u = s_nxt.reveal_lo + tid; u < s_nxt.hi; u += kThreads) a_ring[u & amask] = 0.f;
        __syncthreads();
        const int lo_now = max(0, st.hi - cap);
        const int lo_next = has_next ? max(0, s_nxt.hi - cap) : lo_now;
        for (int so = tid; so < NSO; so += kThreads) {
            const float delta = ((red[so] + red[NSOp + so]) + (red[2 * NSOp + so] + red[3 * NSOp + so]));
            const int col = colof[so];
            const bool entering = pf_n > 0 && col >= pf_e0 && col < pf_e0 + pf_n;
            if (entering) {
                const int e = col - pf_e0;
                float full = 0.f;
                for (int w2 = 0; w2 < kWarps; ++w2) full += wpart[e * kWarps + w2];
                gown[so] = full + delta;
            } else {
                float gv = gown[so] + delta;
                // dictionary rows evicted at t+1 leave the sum
                for (int b = lo_now; b < lo_next && col >= 0; ++b) gv -= a_ring[b & amask] * kval(args, b, col);
                gown[so] = gv;
            }
        }
        // (B4) clear this step's corrections; rows the registers could not serve enter directly
        for (int i = tid; i < st.n_active; i += kThreads) cs[wrap(s0 + i, XS)] = 0.f;
        __syncthreads();
        if (pf_n < 0 && has_next)
            enter_direct(enter_lo(t + 1, s_nxt, st), s_nxt.hi, max(0, s_nxt.hi - cap), s_nxt.hi);
        const TrainStep s3 = load_step(t + 3);
        prefetch(t + 2, s_nn, s_nxt);
        s_cur = s_nxt;
        s_nxt = s_nn;
        s_nn = s3;
        __syncthreads();
    }
    __syncthreads();
    cluster.sync(); // no CTA leaves while a peer may still address its shared memory

    if (*abort_flag) {
        if (tid == 0) atomicExch(args.err, 1);
        return;
    }
    if (rank == 0) {
        const int hi = args.final_hi;
        const int lo = max(0, hi - cap);
        for (int u = lo + tid; u < hi; u += kThreads) a_out[u] = a_ring[u & amask];
        for (int d = tid; d < D; d += kThreads) w_out[d] = w_s[d];
    }
}

int incremental_threads() { return kThreads; }

cudaError_t query_incremental_clusters(int cluster, size_t smem, int users, int* max_clusters)
{
    cudaError_t e = cudaFuncSetAttribute(train_inc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    if (cluster > 8) {
        e = cudaFuncSetAttribute(train_inc_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(unsigned(users * cluster));
    lc.blockDim = dim3(unsigned(kThreads));
    lc.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(max_clusters, train_inc_kernel, &lc);
}

size_t incremental_smem_bytes(int XS, int XP, int NSOp, int A_ring)
{
    return sizeof(float) * (size_t(XS) * NSOp + size_t(XS) * XP + 4 * size_t(XS) + NSOp + size_t(kParts) * NSOp +
                            size_t(A_ring) + kMaxFeatures + kMaxEnter * kWarps) +
           sizeof(int) * (size_t(XS) + NSOp + 1) + 2 * sizeof(uint64_t) + 16;
}

cudaError_t launch_train_incremental(int cluster, size_t smem, cudaStream_t stream, const TrainArgs& args,
                                     int* max_clusters)
{
    cudaError_t e = cudaFuncSetAttribute(train_inc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    if (cluster > 8) {
        e = cudaFuncSetAttribute(train_inc_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(unsigned(args.users * cluster));
    lc.blockDim = dim3(unsigned(kThreads));
    lc.dynamicSmemBytes = smem;
    lc.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    e = cudaOccupancyMaxActiveClusters(max_clusters, train_inc_kernel, &lc);
    if (e != cudaSuccess || *max_clusters < 1) return e;
    return cudaLaunchKernelEx(&lc, train_inc_kernel, args);
}

} // namespace apsm
