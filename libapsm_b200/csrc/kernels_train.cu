// APSM online training on B200: sample packing, per-call kernel-column
// precompute, and the persistent cluster kernel that runs the whole pilot
// sweep in one launch.
//
// Reference behaviour restated here:
//   host step loop          cpp/lib/apsm/apsm_train.cu:100-160
//   per-step kernel         cpp/lib/apsm/apsm_train.cu:271-432
//   prediction f(x_j)       cpp/lib/apsm/apsm_detect.cu:170-226 (+ :131-152)
//   Dedup real embedding    cpp/lib/cuda/cuda_matrix_device.cuh:180-188, 288-296
//
// B200 design (not the reference's): all pilots are known when train() is
// called, so the Gaussian kernel value between a dictionary row u and a
// window row v never changes during the sweep.  gram_columns_kernel computes
// every value the sweep can touch once (wG * exp(ew * ||x_u - x_v||^2), the
// reference's float expression and order) into HBM/L2; the users of one cell
// share it.  The sweep itself is one launch per user: a thread-block cluster
// whose CTAs split the projection window, keep replicated coefficients in
// shared memory, exchange the step's corrections through distributed shared
// memory and meet at one hardware cluster barrier per step (the reference
// pays one cooperative launch plus a grid sync per step).
#include "apsm_kernels.cuh"

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace apsm {

// ---------------------------------------------------------------- packing --

// rx: num_ant x n_total complex (antenna-major), optionally read through a
// sample permutation (trainingShuffle).  Writes real rows
// row0 + 2i (= [Re y_i ; Im y_i]) and row0 + 2i + 1 (= [Im y_i ; -Re y_i]) for
// i < n_total into X (pitch Dp, zero padded), and their squared norms
// (sequential fma, the order of kernel_apsm_detection_linear_original,
// apsm_detect.cu:103-119) into nrm when nrm != nullptr.
__global__ void __launch_bounds__(256) pack_rows_kernel(const float2* __restrict__ rx, int num_ant, int n_total,
                                                        const int* __restrict__ perm, float* __restrict__ X, int Dp,
                                                        int row0, float* __restrict__ nrm)
{
    extern __shared__ float2 tile[]; // [num_ant][kPackSamples]
    const int n0 = blockIdx.x * kPackSamples;
    const int tid = threadIdx.x;
    for (int idx = tid; idx < num_ant * kPackSamples; idx += blockDim.x) {
        int a = idx / kPackSamples, i = idx % kPackSamples;
        int n = n0 + i;
        const int src = (perm != nullptr && n < n_total) ? perm[n] : n;
        tile[idx] = n < n_total ? rx[size_t(a) * n_total + src] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int D = 2 * num_ant;
    const int rows = 2 * kPackSamples;
    for (int idx = tid; idx < rows * Dp; idx += blockDim.x) {
        int r = idx / Dp, d = idx % Dp;
        int i = r >> 1, odd = r & 1;
        if (n0 + i >= n_total) continue;
        float v = 0.f;
        if (d < num_ant) {
            float2 c = tile[d * kPackSamples + i];
            v = odd ? c.y : c.x;
        } else if (d < D) {
            float2 c = tile[(d - num_ant) * kPackSamples + i];
            v = odd ? -c.x : c.y;
        }
        X[size_t(row0 + 2 * (n0 + i) + odd) * Dp + d] = v;
    }
    if (nrm != nullptr && tid < rows) {
        int i = tid >> 1, odd = tid & 1;
        if (n0 + i < n_total) {
            float acc = 0.f;
            for (int d = 0; d < D; ++d) {
                float v;
                if (d < num_ant) {
                    float2 c = tile[d * kPackSamples + i];
                    v = odd ? c.y : c.x;
                } else {
                    float2 c = tile[(d - num_ant) * kPackSamples + i];
                    v = odd ? -c.x : c.y;
                }
                acc = fmaf(v, v, acc);
            }
            nrm[row0 + 2 * (n0 + i) + odd] = acc;
        }
    }
}

// y[u * y_stride + row0 + 2i + {0,1}] = (re, im) of tx[u * P + perm[i]]
// (targets of the Dedup rows: column 2n -> Re x_n, 2n+1 -> Im x_n).
__global__ void gather_targets_kernel(const float2* __restrict__ tx, int P, int users, const int* __restrict__ perm,
                                      float* __restrict__ y, size_t y_stride, int row0)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P * users) return;
    const int u = i / P, n = i % P;
    const float2 v = tx[size_t(u) * P + (perm ? perm[n] : n)];
    y[size_t(u) * y_stride + row0 + 2 * n] = v.x;
    y[size_t(u) * y_stride + row0 + 2 * n + 1] = v.y;
}

// ------------------------------------------------------- kernel columns --

// Column v of K holds wG * exp(ew * ||x_u - x_v||^2) for universe rows
// u = ubase(v) + i, i < Lk, where ubase(v) = max(0, v + 1 - cap) rounded down
// to a multiple of 4 (16-byte aligned columns).  That covers every dictionary
// row visible while row v sits in a projection window (u in [v + 1 - cap,
// v + q2)).  Entries with u >= nU are 0 and never read.  Arithmetic is the
// reference's: sequential fma of (d_u - x_v)^2, float product with the exp
// weight, expf, product with the Gaussian weight (apsm_detect.cu:131-152,
// apsm_train.cu:219).
__global__ void __launch_bounds__(256) gram_columns_kernel(const float* __restrict__ X, int Dp, int D, int nU,
                                                           int v_first, int nV, int Lk, int cap, ModelParams mp,
                                                           float* __restrict__ K)
{
    __shared__ float xv[kGramColsPerBlock][kMaxFeatures];
    const int vb = v_first + blockIdx.y * kGramColsPerBlock;
    for (int idx = threadIdx.x; idx < kGramColsPerBlock * D; idx += blockDim.x) {
        int c = idx / D, d = idx % D;
        int v = vb + c;
        xv[c][d] = (v < v_first + nV) ? X[size_t(v) * Dp + d] : 0.f;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Lk) return;
    for (int c = 0; c < kGramColsPerBlock; ++c) {
        const int v = vb + c;
        if (v >= v_first + nV) break;
        const int u = column_base(v, cap) + i;
        float val = 0.f;
        if (u < nU) {
            const float* xu = X + size_t(u) * Dp;
            float acc = 0.f;
            for (int d = 0; d < D; ++d) {
                float diff = __ldg(xu + d) - xv[c][d];
                acc = fmaf(diff, diff, acc);
            }
            val = __fmul_rn(mp.wG, expf(__fmul_rn(mp.ew, acc)));
        }
        K[size_t(v - v_first) * Lk + i] = val;
    }
}

// ---------------------------------------------------------- the sweep ----

namespace {

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src)
{
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gmem_src) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Optional phase timestamps (build with -DAPSM_TRAIN_PROFILE): thread 0 of the
// first CTA records %globaltimer at fixed points of each step into args.prof.
#ifdef APSM_TRAIN_PROFILE
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
#define APSM_PROF_MARK(k)                                                                     \
    if (args.prof != nullptr && blockIdx.x == 0 && tid == 0 && t < kProfSteps)                \
        args.prof[size_t(t) * kProfMarks + (k)] = global_ns();
#else
#define APSM_PROF_MARK(k)
#endif

} // namespace

// Shared memory carve-up of train_exact_kernel (floats):
//   a_ring [A_ring]         coefficients of the visible rows, replicated per CTA
//   w_s    [128]            linear weights, replicated per CTA
//   cbuf   [2][q2]          step corrections, written by their owner into every CTA
//   red    [nwarps][32]     lane partials of the predictions
//   xw     [XW][Dp]         rows of the projection window (and the next kLookahead steps)
//   yw, nw [XW]             their targets and squared norms
//   kcol   [NS][Lc]         kernel columns of the window rows this CTA owns (kStaged)
//
// Window row v is owned by CTA v % C for as long as it stays in the window.
// Rows, targets, norms and owned kernel columns for step t + kLookahead are
// fetched with cp.async while step t computes; step t waits only for its own
// group.  cp.async completion is tracked by the hardware (no spin loops).
template <bool kStaged>
__global__ void __launch_bounds__(1024) train_exact_kernel(TrainArgs args)
{
    cg::cluster_group cluster = cg::this_cluster();
    const int C = int(cluster.num_blocks());
    const int rank = int(cluster.block_rank());
    const int user = blockIdx.x / C;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nthreads = blockDim.x, nwarps = nthreads >> 5;

    extern __shared__ __align__(16) float smem[];
    float* xw = smem;                          // 16-byte aligned rows first
    float* kcol = xw + size_t(args.XW) * args.Dp;
    float* a_ring = kcol + (kStaged ? size_t(args.NS) * args.Lc : 0);
    float* w_s = a_ring + args.A_ring;
    float* cbuf = w_s + kMaxFeatures;
    float* red = cbuf + 2 * args.q2;
    float* yw = red + nwarps * 32;
    float* nw = yw + args.XW;

    const int D = args.D, Dp = args.Dp, cap = args.cap, q2 = args.q2;
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
                const int r = r0 + idx / q4, c4 = idx - (idx / q4) * q4;
                cp_async16(xw + (r & xmask) * Dp + 4 * c4, X + size_t(r) * Dp + 4 * c4);
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
                    const int len4 = (round_up(uint32_t(min(args.nU, v + q2)), 4u) - ub) >> 2;
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
    cluster.sync(); // every CTA resident before the first remote write

#pragma unroll 1
    for (int t = 0; t < n_steps; ++t) {
        APSM_PROF_MARK(0);
        cp_async_wait<kLookahead - 1>(); // this step's rows and columns have landed
        __syncthreads();
        APSM_PROF_MARK(1);

        const TrainStep st = sv[0];
        const int lo = max(0, st.hi - cap);
        const int M = st.hi - lo;
        const int start = st.hi - st.wk;
        float* cb = cbuf + (t & 1) * q2;

        // predictions with the pre-step coefficients; this CTA owns window rows v % C == rank
        const int first = start + ((rank - start % C) + C) % C;
        for (int v = first + C * warp; v < start + st.n_active; v += C * nwarps) {
            const int ub = column_base(v, cap);
            const float* kc = kStaged ? kcol + size_t((v / C) % args.NS) * args.Lc - ub
                                      : K + size_t(v - args.v_first) * args.Lk - ub;
            const float* xv = xw + (v & xmask) * Dp;
            float p = 0.f;
            int b = lane;
            // kernel_apsm_detection_original order: per b the linear term, then the Gaussian term
            for (; b < D; b += 32) {
                p = __fadd_rn(p, __fmul_rn(__fmul_rn(mp.wL, xv[b]), w_s[b]));
                if (b < M) p = __fadd_rn(p, __fmul_rn(kStaged ? kc[lo + b] : __ldg(kc + lo + b), a_ring[(lo + b) & amask]));
            }
            // Gaussian-only tail in chunks of 8: all loads first, then the ordered sum.
            // Past the end the product is +0, and p + (+0) == p for the p this sum can reach.
            for (; b < M; b += 8 * 32) {
                float kv[8], av[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int bb = b + 32 * j;
                    const bool ok = bb < M;
                    kv[j] = ok ? (kStaged ? kc[lo + bb] : __ldg(kc + lo + bb)) : 0.f;
                    av[j] = ok ? a_ring[(lo + bb) & amask] : 0.f;
                }
#pragma unroll
                for (int j = 0; j < 8; ++j) p = __fadd_rn(p, __fmul_rn(kv[j], av[j]));
            }
            red[warp * 32 + lane] = p;
            __syncwarp();
            if (lane == 0) {
                float part[32];
#pragma unroll
                for (int l = 0; l < 32; ++l) part[l] = red[warp * 32 + l];
                float f = part[0];
#pragma unroll
                for (int l = 1; l < 32; ++l) f = __fadd_rn(f, part[l]);
                // hyperslab projection (apsm_train.cu:380-401)
                const float e = __fsub_rn(yw[v & xmask], f);
                float c = 0.f;
                if (e > mp.eB) c = __fsub_rn(e, mp.eB);
                else if (e < -mp.eB) c = __fadd_rn(e, mp.eB);
                const float linearNorm = __fmul_rn(mp.wL, nw[v & xmask]);
                c = __fdiv_rn(c, float(st.wk));
                c = __fdiv_rn(c, __fadd_rn(linearNorm, mp.wG));
                for (int r = 0; r < C; ++r) *cluster.map_shared_rank(cb + (v - start), r) = c;
            }
            __syncwarp();
        }
        APSM_PROF_MARK(2);
        // Split cluster barrier: the release publishes this CTA's corrections;
        // work that does not read them overlaps the wait.
        asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
        issue(t + kLookahead, sv[kLookahead]);
        // rows revealed by the next step start with a = 0 (not visible at this step)
        for (int u = sv[1].reveal_lo + tid; u < sv[1].hi; u += nthreads) a_ring[u & amask] = 0.f;
        const TrainStep next = load_step(t + kLookahead + 2);
        APSM_PROF_MARK(3);
        asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
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
                        xv4[j] = xw[((start + i + j * kWGroups) & xmask) * Dp + d];
                    }
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc = __fadd_rn(acc, __fmul_rn(cv[j], xv4[j]));
                }
                for (; i < st.n_active; i += kWGroups)
                    acc = __fadd_rn(acc, __fmul_rn(cb[i], xw[((start + i) & xmask) * Dp + d]));
            }
            acc = __fadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, 1));
            acc = __fadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, 2));
            acc = __fadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, 4));
            if (d < D && g == 0) w_s[d] = __fadd_rn(w_s[d], acc);
        }
#pragma unroll
        for (int k = 0; k < kLookahead + 1; ++k) sv[k] = sv[k + 1];
        sv[kLookahead + 1] = next;
        APSM_PROF_MARK(5);
    }
    cp_async_wait<0>();
    __syncthreads();

    // write back: coefficients of the rows visible after the sweep, and w
    if (rank == 0) {
        const int hi = args.final_hi;
        const int lo = max(0, hi - cap);
        for (int u = lo + tid; u < hi; u += nthreads) a_out[u] = a_ring[u & amask];
        for (int d = tid; d < D; d += nthreads) w_out[d] = w_s[d];
    }
}

cudaError_t launch_train_exact(bool staged, int cluster, int threads, size_t smem, cudaStream_t stream,
                               const TrainArgs& args, int* max_clusters)
{
    auto kern = staged ? train_exact_kernel<true> : train_exact_kernel<false>;
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

} // namespace apsm
