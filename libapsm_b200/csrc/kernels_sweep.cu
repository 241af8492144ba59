// APSM training sweep on B200: the whole pilot sequence in one launch.
//
// Reference behaviour restated (cpp/lib/apsm/apsm_train.cu:100-166 host loop,
// :271-432 kernel, cpp/lib/apsm/apsm_detect.cu:170-226 prediction): at each
// step every window row j is predicted with the pre-step coefficients,
//   f_j = sum_b [b < D] (wL x_j[b]) w[b]  +  [b < M] (wG k(d_b, x_j)) a_b
// (lane l of 32 accumulates b = l, l+32, ... in order; the 32 partials are
// added sequentially), projected onto the hyperslab
//   c_j = sign(e) max(|e| - eB, 0) / Wk / (wL ||x_j||^2 + wG),  e = y_j - f_j,
// and then a_j += c_j, w += sum_j c_j x_j.
//
// B200 design: one thread-block cluster per user runs all steps.  Window row
// v belongs to CTA v % C; that CTA keeps its kernel column (precomputed by
// gram_columns_kernel) in shared memory, fetched with cp.async a few steps
// before it is needed together with the row, its target and its norm.  The
// coefficients and linear weights are replicated in every CTA's shared
// memory.  A step's corrections c_j are pushed to every CTA of the cluster
// with st.async into its shared memory; each CTA's mbarrier completes when
// all n_active corrections of the step have landed (complete_tx), so CTAs
// synchronise through the data itself, with no cluster-wide barrier per step.
// Every wait is bounded (2 s); on expiry the kernel records an error in
// args.err and all CTAs leave the sweep.
#include "apsm_kernels.cuh"

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace apsm {

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(smem_dst)), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

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

__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, uint32_t parity)
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

constexpr unsigned long long kWaitLimitNs = 2000000000ull; // 2 s

// Bounded wait for a phase of a barrier fed by st.async from the cluster.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    if (mbar_try_wait_cluster(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        for (int i = 0; i < 256; ++i)
            if (mbar_try_wait_cluster(bar, parity)) return true;
        if (global_ns() - t0 > kWaitLimitNs) return false;
    }
}

// st.async of one float into CTA `rank`'s shared memory at the address that
// `local` has here, completing 4 bytes of transaction on that CTA's `bar`.
__device__ __forceinline__ void st_async_f32(const float* local, const uint64_t* bar, uint32_t rank, float v)
{
    uint32_t raddr, rbar;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(raddr) : "r"(smem_u32(local)), "r"(rank));
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(rbar) : "r"(smem_u32(bar)), "r"(rank));
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];" ::"r"(raddr),
                 "r"(__float_as_uint(v)), "r"(rbar)
                 : "memory");
}

#ifdef APSM_TRAIN_PROFILE
#define APSM_PROF_MARK(k)                                                                     \
    if (args.prof != nullptr && blockIdx.x == 0 && tid == 0 && t < kProfSteps)                \
        args.prof[size_t(t) * kProfMarks + (k)] = global_ns();
#else
#define APSM_PROF_MARK(k)
#endif

} // namespace

// Shared memory carve-up (floats, then two mbarriers):
//   xw     [XW][XP]   window rows (and the next kLookahead steps' rows), XP = Dp + 4
//   kcol   [NS][Lc]   kernel columns of the window rows this CTA owns (kStaged)
//   a_ring [A_ring]   coefficients of the visible rows, replicated per CTA
//   w_s    [128]      linear weights, replicated per CTA
//   cbuf   [2][q2]    the step's corrections (st.async from their owner CTAs)
//   red    [nwarps][32] lane partials of the predictions
//   yw, nw [XW]       targets and squared norms of the window rows
//   nbuf   [2][16]    normConstraint: the CTAs' partial sums of ||f_G||^2 (st.async)
//   npart  [32]       normConstraint: warp partials
// kGlobA: dictionaries whose coefficient ring does not fit shared memory keep it
// in global memory instead, one private copy per CTA (args.a_glob, A_ring floats
// per CTA): every CTA still applies every correction to its own copy, so no
// copy is read by another CTA.
template <bool kStaged, bool kGlobA>
__global__ void __launch_bounds__(1024) train_sweep_kernel(TrainArgs args)
{
    cg::cluster_group cluster = cg::this_cluster();
    const int C = int(cluster.num_blocks());
    const int rank = int(cluster.block_rank());
    const int user = blockIdx.x / C;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nthreads = blockDim.x, nwarps = nthreads >> 5;

    const int D = args.D, Dp = args.Dp, XP = args.XP, cap = args.cap, q2 = args.q2;
    extern __shared__ __align__(16) float smem[];
    float* xw = smem;
    float* kcol = xw + size_t(args.XW) * XP;
    float* a_smem = kcol + (kStaged ? size_t(args.NS) * args.Lc : 0);
    float* a_ring = kGlobA ? args.a_glob + size_t(blockIdx.x) * args.A_ring : a_smem;
    float* w_s = a_smem + (kGlobA ? 0 : args.A_ring);
    float* cbuf = w_s + kMaxFeatures;
    float* red = cbuf + 2 * q2;
    float* yw = red + nwarps * 32;
    float* nw = yw + args.XW;
    float* nbuf = nw + args.XW;
    float* npart = nbuf + 32;
    uint64_t* cfull = reinterpret_cast<uint64_t*>(npart + 32); // [2] corrections
    uint64_t* nfull = cfull + 2;                               // [2] normConstraint partials
    volatile int* abort_flag = reinterpret_cast<volatile int*>(cfull + 4);

    const int amask = args.A_ring - 1, xmask = args.XW - 1;
    const int n_steps = args.n_steps;
    const float* __restrict__ X = args.X;
    const float* __restrict__ nrm = args.nrm;
    const float* __restrict__ K = args.K;
    const float* __restrict__ y = args.y + size_t(user) * args.y_stride;
    float* __restrict__ a_out = args.a + size_t(user) * args.a_stride;
    float* __restrict__ w_out = args.w + size_t(user) * D;
    const ModelParams mp = args.mp;

    int rows_hi = 0, cols_hi = 0;
    auto issue = [&](int tt, const TrainStep& st) {
        if (tt < n_steps) {
            const int start = st.hi - st.wk;
            const int r0 = max(rows_hi, start), r1 = st.hi;
            const int q4 = Dp >> 2;
            for (int idx = tid; idx < (r1 - r0) * q4; idx += nthreads) {
                const int rr = idx / q4;
                const int r = r0 + rr, c4 = idx - rr * q4;
                cp_async16(xw + (r & xmask) * XP + 4 * c4, X + size_t(r) * Dp + 4 * c4);
            }
            for (int r = r0 + tid; r < r1; r += nthreads) {
                cp_async4(yw + (r & xmask), y + r);
                cp_async4(nw + (r & xmask), nrm + r);
            }
            rows_hi = max(rows_hi, r1);
            if (kStaged) {
                const int c0 = max(cols_hi, start), c1 = st.hi;
                for (int v = c0 + ((rank - c0 % C) + C) % C; v < c1; v += C) {
                    const int ub = column_base(v, cap);
                    const int len4 = (int(round_up(uint32_t(min(args.nU, v + q2)), 4u)) - ub) >> 2;
                    float* dst = kcol + size_t((v / C) % args.NS) * args.Lc;
                    const float* src = K + size_t(v - args.v_first) * args.Lk;
                    for (int idx = tid; idx < len4; idx += nthreads) cp_async16(dst + 4 * idx, src + 4 * idx);
                }
                cols_hi = max(cols_hi, c1);
            }
        }
        cp_async_commit();
    };
    auto load_step = [&](int tt) -> TrainStep {
        return tt < n_steps ? args.steps[tt] : TrainStep{0, 0, 0, 0};
    };

    if (tid == 0) {
        mbar_init(&cfull[0], 1);
        mbar_init(&cfull[1], 1);
        mbar_init(&nfull[0], 1);
        mbar_init(&nfull[1], 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // Rows already in the dictionary before this call (all visible: used_before <= cap).
    for (int u = tid; u < args.used_before; u += nthreads) a_ring[u & amask] = a_out[u];
    for (int d = tid; d < kMaxFeatures; d += nthreads) w_s[d] = d < D ? w_out[d] : 0.f;
    // sv[k] = step t + k, kept in registers so no step waits on a global load
    TrainStep sv[kLookahead + 2];
#pragma unroll
    for (int k = 0; k < kLookahead + 2; ++k) sv[k] = load_step(k);
    if (n_steps > 0)
        for (int u = sv[0].reveal_lo + tid; u < sv[0].hi; u += nthreads) a_ring[u & amask] = 0.f;
#pragma unroll
    for (int k = 0; k < kLookahead; ++k) issue(k, sv[k]);
    cluster.sync(); // every CTA resident and its barriers initialised before the first st.async

#pragma unroll 1
    for (int t = 0; t < n_steps; ++t) {
        APSM_PROF_MARK(0);
        cp_async_wait<kLookahead - 1>(); // this step's rows and columns have landed
        __syncthreads();
        if (*abort_flag) break; // uniform: read after the block barrier
        APSM_PROF_MARK(1);

        const TrainStep st = sv[0];
        const int lo = max(0, st.hi - cap);
        const int M = st.hi - lo;
        const int start = st.hi - st.wk;
        float* cb = cbuf + (t & 1) * q2;
        uint64_t* bar = &cfull[t & 1];
        if (tid == 0) mbar_expect_tx(bar, uint32_t(st.n_active) * 4u);
        if (tid == 0 && args.norm_c > 0.f) mbar_expect_tx(&nfull[t & 1], uint32_t(C) * 4u);

        // predictions with the pre-step coefficients; this CTA owns window rows v % C == rank
        const int first = start + ((rank - start % C) + C) % C;
        for (int v = first + C * warp; v < start + st.n_active; v += C * nwarps) {
            const int ub = column_base(v, cap);
            const float* kc = kStaged ? kcol + size_t((v / C) % args.NS) * args.Lc - ub
                                      : K + size_t(v - args.v_first) * args.Lk - ub;
            const float* xv = xw + (v & xmask) * XP;
            float p = 0.f;
            int b = lane;
            // kernel_apsm_detection_original order: per b the linear term, then the Gaussian term
            for (; b < D; b += 32) {
                p = __fadd_rn(p, __fmul_rn(__fmul_rn(mp.wL, xv[b]), w_s[b]));
                if (b < M) p = __fadd_rn(p, __fmul_rn(kStaged ? kc[lo + b] : __ldg(kc + lo + b), a_ring[(lo + b) & amask]));
            }
            // Gaussian-only tail in chunks of 8: all loads first, then the ordered sum.  Rows
            // lo + b sit at ring positions (lo & amask) + b until the ring wraps at b = bw, then
            // at b - bw: whole chunks on either side of the wrap index both arrays directly
            // (no masks, no range checks); the chunk across the wrap and the last one are
            // checked, where past the end the product is +0, and p + (+0) == p for the p this
            // sum can reach.
            const float* kp = kc + lo;
            const int lo_m = lo & amask, bw = args.A_ring - lo_m;
            auto chunk_direct = [&](const float* ap) {
                float kv[8], av[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    kv[j] = kStaged ? kp[b + 32 * j] : __ldg(kp + b + 32 * j);
                    av[j] = ap[b + 32 * j];
                }
#pragma unroll
                for (int j = 0; j < 8; ++j) p = __fadd_rn(p, __fmul_rn(kv[j], av[j]));
            };
            auto chunk_checked = [&]() {
                float kv[8], av[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int bb = b + 32 * j;
                    const bool ok = bb < M;
                    kv[j] = ok ? (kStaged ? kp[bb] : __ldg(kp + bb)) : 0.f;
                    av[j] = ok ? a_ring[(lo + bb) & amask] : 0.f;
                }
#pragma unroll
                for (int j = 0; j < 8; ++j) p = __fadd_rn(p, __fmul_rn(kv[j], av[j]));
            };
            const int lim1 = min(M, bw);
            for (; b + 7 * 32 < lim1; b += 8 * 32) chunk_direct(a_ring + lo_m);
            if (b < lim1) { // the chunk that reaches the wrap or the end
                chunk_checked();
                b += 8 * 32;
            }
            for (; b + 7 * 32 < M; b += 8 * 32) chunk_direct(a_ring - bw); // past the wrap: b >= bw
            for (; b < M; b += 8 * 32) chunk_checked();
            if (v == first) APSM_PROF_MARK(6);
            red[warp * 32 + lane] = p;
            __syncwarp();
            float c = 0.f;
            if (lane == 0) {
                const float4* r4 = reinterpret_cast<const float4*>(red + warp * 32);
                float f = 0.f;
#pragma unroll
                for (int l4 = 0; l4 < 8; ++l4) {
                    const float4 q = r4[l4];
                    f = (l4 == 0) ? q.x : __fadd_rn(f, q.x);
                    f = __fadd_rn(f, q.y);
                    f = __fadd_rn(f, q.z);
                    f = __fadd_rn(f, q.w);
                }
                // hyperslab projection (apsm_train.cu:380-401)
                const float e = __fsub_rn(yw[v & xmask], f);
                if (e > mp.eB) c = __fsub_rn(e, mp.eB);
                else if (e < -mp.eB) c = __fadd_rn(e, mp.eB);
                const float linearNorm = __fmul_rn(mp.wL, nw[v & xmask]);
                c = __fdiv_rn(c, float(st.wk));
                c = __fdiv_rn(c, __fadd_rn(linearNorm, mp.wG));
            }
            if (v == first) APSM_PROF_MARK(7);
            c = __shfl_sync(0xffffffffu, c, 0);
            if (lane < C) st_async_f32(cb + (v - start), bar, uint32_t(lane), c);
            __syncwarp();
        }
        APSM_PROF_MARK(2);
        // work that does not need this step's corrections
        issue(t + kLookahead, sv[kLookahead]);
        // rows revealed by the next step start with a = 0 (not visible at this step)
        for (int u = sv[1].reveal_lo + tid; u < sv[1].hi; u += nthreads) a_ring[u & amask] = 0.f;
        const TrainStep next = load_step(t + kLookahead + 2);
        APSM_PROF_MARK(3);
        if (!mbar_wait_bounded(bar, uint32_t(t >> 1) & 1u)) *abort_flag = 1;
        APSM_PROF_MARK(4);

        // a_j += c_j (apsm_train.cu:407)
        for (int i = tid; i < st.n_active; i += nthreads) {
            float* ap = a_ring + ((start + i) & amask);
            *ap = __fadd_rn(*ap, cb[i]);
        }
        // w += sum_j c_j x_j (apsm_train.cu:413-428) in the fixed group order:
        // group g sums window positions i = g, g+8, ... ascending, groups combine
        // as ((g0+g1)+(g2+g3))+((g4+g5)+(g6+g7)).  A zero correction adds +0
        // (acc starts at +0 and cannot become -0), i.e. nothing.
        const int nwork = int(round_up(uint32_t(D * kWGroups), 32u));
        for (int idx = tid; idx < nwork; idx += nthreads) {
            const int d = idx / kWGroups, g = idx % kWGroups;
            float acc = 0.f;
            if (d < D) {
                int i = g;
                for (; i + 3 * kWGroups < st.n_active; i += 4 * kWGroups) {
                    float cv[4], xv4[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        cv[j] = cb[i + j * kWGroups];
                        xv4[j] = xw[((start + i + j * kWGroups) & xmask) * XP + d];
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc = __fadd_rn(acc, __fmul_rn(cv[j], xv4[j]));
                }
                for (; i < st.n_active; i += kWGroups)
                    acc = __fadd_rn(acc, __fmul_rn(cb[i], xw[((start + i) & xmask) * XP + d]));
            }
            acc = __fadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, 1));
            acc = __fadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, 2));
            acc = __fadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, 4));
            if (d < D && g == 0) w_s[d] = __fadd_rn(w_s[d], acc);
        }
        if (args.norm_c > 0.f) {
            // normConstraint (kernel_adapt_coeffs, apsm_train.cu:190-256): ||f_G||^2 =
            // sum_v a_v (wG a_v + 2 sum_{u<v} K(u, v) a_u) over the dictionary [lo, hi), column v of
            // K holding K(u, v) for its older rows; CTA r takes the columns v = r mod C.  The CTAs'
            // partials go to every CTA (st.async), each adds them in rank order, so all CTAs see
            // the same norm and scale their copies of the coefficients alike.
            __syncthreads(); // this step's a_j are final
            const int lo = max(0, st.hi - cap);
            float acc = 0.f;
            for (int v = lo + ((rank - lo % C) + C) % C + C * warp; v < st.hi; v += C * nwarps) {
                const float* kc = K + size_t(v - args.v_first) * args.Lk - column_base(v, cap);
                float sv = 0.f;
                for (int u = lo + lane; u < v; u += 32) sv = fmaf(__ldg(kc + u), a_ring[u & amask], sv);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) sv += __shfl_xor_sync(0xffffffffu, sv, o);
                const float av = a_ring[v & amask];
                acc = fmaf(av, fmaf(2.f, sv, mp.wG * av), acc);
            }
            if (lane == 0) npart[warp] = acc;
            __syncthreads();
            if (warp == 0) {
                float x = lane < nwarps ? npart[lane] : 0.f;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                if (lane < C) st_async_f32(nbuf + (t & 1) * 16 + rank, &nfull[t & 1], uint32_t(lane), x);
            }
            if (!mbar_wait_bounded(&nfull[t & 1], uint32_t(t >> 1) & 1u)) *abort_flag = 1;
            float norm = 0.f;
            for (int r = 0; r < C; ++r) norm += nbuf[(t & 1) * 16 + r];
            if (norm > 0.f) norm = sqrtf(norm);
            float factor = 1.f;
            if (norm > args.norm_c) {
                factor = __fdiv_rn(args.norm_c, norm);
                for (int u = lo + tid; u < st.hi; u += nthreads) a_ring[u & amask] = __fmul_rn(a_ring[u & amask], factor);
            }
            if (args.snap_scale && rank == 0 && tid == 0) args.snap_scale[size_t(user) * n_steps + t] = factor;
            if (!args.snap_a) __syncthreads(); // scaled coefficients visible before the next step
        }
        if (args.snap_a) {
            // training history: the model after this step (every CTA holds the same copy)
            __syncthreads();
            if (rank == 0) {
                float* sa = args.snap_a + (size_t(user) * n_steps + t) * q2;
                for (int i = tid; i < st.n_active; i += nthreads) sa[i] = a_ring[(start + i) & amask];
                float* sw = args.snap_w + (size_t(user) * n_steps + t) * D;
                for (int d = tid; d < D; d += nthreads) sw[d] = w_s[d];
            }
        }
#pragma unroll
        for (int k = 0; k < kLookahead + 1; ++k) sv[k] = sv[k + 1];
        sv[kLookahead + 1] = next;
        APSM_PROF_MARK(5);
    }
    cp_async_wait<0>();
    __syncthreads();
    cluster.sync(); // no CTA leaves while a peer may still address its shared memory

    if (*abort_flag) {
        if (tid == 0) atomicExch(args.err, 1);
        return;
    }
    // write back: coefficients of the rows visible after the sweep, and w
    if (rank == 0) {
        const int hi = args.final_hi;
        const int lo = max(0, hi - cap);
        for (int u = lo + tid; u < hi; u += nthreads) a_out[u] = a_ring[u & amask];
        for (int d = tid; d < D; d += nthreads) w_out[d] = w_s[d];
    }
}

namespace {
using SweepKernel = void (*)(TrainArgs);
SweepKernel sweep_kernel(bool staged, bool glob_a)
{
    if (glob_a) return staged ? train_sweep_kernel<true, true> : train_sweep_kernel<false, true>;
    return staged ? train_sweep_kernel<true, false> : train_sweep_kernel<false, false>;
}
} // namespace

cudaError_t launch_train_exact(bool staged, int cluster, int threads, size_t smem, cudaStream_t stream,
                               const TrainArgs& args, int* max_clusters)
{
    auto kern = sweep_kernel(staged, args.a_glob != nullptr);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    if (cluster > 8) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(unsigned(args.users * cluster));
    lc.blockDim = dim3(unsigned(threads));
    lc.dynamicSmemBytes = smem;
    lc.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    e = cudaOccupancyMaxActiveClusters(max_clusters, kern, &lc);
    if (e != cudaSuccess) return e;
    if (*max_clusters < 1) return cudaSuccess; // caller reports it
    return cudaLaunchKernelEx(&lc, kern, args);
}

cudaError_t query_train_clusters(bool staged, bool glob_a, int cluster, int threads, size_t smem, int users,
                                 int* max_clusters)
{
    auto kern = sweep_kernel(staged, glob_a);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    if (cluster > 8) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(unsigned(users * cluster));
    lc.blockDim = dim3(unsigned(threads));
    lc.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(max_clusters, kern, &lc);
}

} // namespace apsm
