// Kernel columns of the batched training sweep on the tensor cores (tcgen05).
//
// Same quantities as batch_kcol_kernel (kernels_batch_kcol.cu): for every pair
// n entering a window, column n holds against every pair b the sweep combines
// it with (b in [max(0, n + 1 - capP), min(n + qP, nP))) the combined kernel
// values (A + wL r, Bp + wL m, Bm - wL m) with r + i m = y_b^H y_n -- the
// reference's distance loop and linear kernel (cpp/lib/apsm/apsm_detect.cu:
// 103-152) formed from y_b^H y_n and the pair norms.  The cross terms y_b^H y_n
// of a band of the job's Gram matrix are UMMAs here instead of 4N scalar FMAs
// per entry: TF32 operands split hi + lo, three products per K step (the
// split's cross terms carry ~2^-21 of |y_b||y_n|, FP32 accuracy), FP32
// accumulation in tensor memory.
//
// One CTA owns a chunk of 64 column pairs n (the fixed B operand: rows 2j =
// [Re y_n; Im y_n], 2j+1 = [-Im y_n; Re y_n], UMMA N = 128) and streams the
// 128-pair row tiles of its band (A operand: rows [Re y_b; Im y_b], UMMA
// M = 128).  Accumulator column 2j of row b holds Re(y_n^H y_b) = r and
// column 2j+1 holds Im(y_n^H y_b) = -m.  The epilogue lane owns row b, so for
// one column n the 32 lanes of a warp store 32 consecutive float4 entries.
//
// Roles (320 threads): warps 0-7 epilogue (warp w: TMEM lanes 32 (w % 4)..,
// column half w / 4), warp 8 producer (bulk copies of the column chunk, the
// row tiles and their norms), warp 9 TMEM allocator and MMA issuer.  Every
// mbarrier wait is bounded; on expiry the CTA records an error, still waits
// for its own copies and products, releases tensor memory and returns.
#include "apsm_batch.cuh"
#include "apsm_tc.cuh"

#include <algorithm>

namespace apsm {

namespace {

using namespace tc;

constexpr int kMode = kTF32x3;
constexpr int kRowTile = 128;  // rows b per streamed tile (UMMA M)
constexpr int kColPairs = 64;  // column pairs n per CTA
constexpr int kColN = 128;     // accumulator columns per tile (UMMA N)
constexpr int kEpiWarps = 8;
constexpr int kThreads = (kEpiWarps + 2) * 32;
constexpr int kStages = 2;

__host__ __device__ constexpr size_t op_bytes(int R, int Kp) { return size_t(R) * 2 * Kp * 4; } // TF32 hi | lo

// A row tiles (pairs b of [0, nP)) and B column chunks (pairs n of [n_first, nP)) of every
// job, plus the row tiles' norms; blockIdx.x < a_tiles: row tile, else column chunk.
__global__ void __launch_bounds__(256) kcol_tc_pack_kernel(const BatchKcolTcJob* __restrict__ jobs)
{
    using T = OpTraits<kMode>;
    const BatchKcolTcJob& jb = jobs[blockIdx.y];
    const int u = blockIdx.x;
    if (u >= jb.a_tiles + jb.b_chunks) return;
    const bool row_tile = u < jb.a_tiles;
    const int Kp = jb.Kp, N = jb.N, Np = jb.Np;
    const int nchunk = Kp / T::kChunk; // 16-byte K chunks of the hi half
    uint8_t* tile = row_tile ? jb.a_ops + size_t(u) * op_bytes(kRowTile, Kp)
                             : jb.b_ops + size_t(u - jb.a_tiles) * op_bytes(kColN, Kp);
    for (int idx = threadIdx.x; idx < 128 * nchunk; idx += blockDim.x) {
        const int r = idx % 128, c = idx / 128;
        int p;          // pair of this row
        bool rot = false; // row [-Im y; Re y]
        if (row_tile) {
            p = u * kRowTile + r;
        } else {
            p = jb.n_first + (u - jb.a_tiles) * kColPairs + (r >> 1);
            rot = (r & 1) != 0;
        }
        uint32_t hw[4], lw[4];
#pragma unroll
        for (int e = 0; e < T::kChunk; ++e) {
            const int k = c * T::kChunk + e;
            float x = 0.f;
            if (p < jb.nP && k < 2 * N) {
                const float2 v = jb.Y[size_t(p) * Np + (k < N ? k : k - N)];
                x = !rot ? (k < N ? v.x : v.y) : (k < N ? -v.y : v.x);
            }
            float hi, lo;
            split_operand<kMode>(x, &hi, &lo);
            hw[e] = __float_as_uint(hi);
            lw[e] = __float_as_uint(lo);
        }
        const size_t off = size_t(c) * (128 * 16) + (r >> 3) * 128 + (r & 7) * 16;
        *reinterpret_cast<uint4*>(tile + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        *reinterpret_cast<uint4*>(tile + size_t(nchunk) * (128 * 16) + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
    }
    if (row_tile)
        for (int r = threadIdx.x; r < kRowTile; r += blockDim.x) {
            const int b = u * kRowTile + r;
            jb.a_nrm[size_t(u) * kRowTile + r] = b < jb.nP ? jb.nrm[b] : 0.f;
        }
}

__global__ void __launch_bounds__(kThreads, 1)
    kcol_tc_kernel(const BatchKcolTcJob* __restrict__ jobs, int n_jobs, const int* __restrict__ chunk_prefix,
                   int Kpmax, BatchCommon cm, int* err, unsigned long long wait_ns)
{
    using T = OpTraits<kMode>;
    // job of this CTA: chunk_prefix[j] <= blockIdx.x < chunk_prefix[j + 1]
    int lo = 0, hi = n_jobs;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (chunk_prefix[mid] <= int(blockIdx.x)) lo = mid;
        else hi = mid;
    }
    const BatchKcolTcJob& jb = jobs[lo];
    const int ci = int(blockIdx.x) - chunk_prefix[lo];
    const int nP = jb.nP, capP = jb.capP, qP = cm.qP;
    const int n0 = jb.n_first + ci * kColPairs;
    const int n_last = min(n0 + kColPairs, nP) - 1;
    const int b_lo = col_begin(n0, capP), b_hi = col_end(n_last, qP, nP);
    const int t0 = b_lo / kRowTile, t1 = (b_hi + kRowTile - 1) / kRowTile; // row tiles of the band
    const int ntile = max(0, t1 - t0);

    extern __shared__ __align__(1024) uint8_t smem[];
    const uint32_t a_bytes = uint32_t(op_bytes(kRowTile, jb.Kp));
    const uint32_t b_bytes = uint32_t(op_bytes(kColN, jb.Kp));
    const uint32_t a_stride = uint32_t(op_bytes(kRowTile, Kpmax));
    uint8_t* sB = smem;                                   // the column chunk
    uint8_t* sA = sB + op_bytes(kColN, Kpmax);            // [kStages] row tiles
    float* sN = reinterpret_cast<float*>(sA + size_t(kStages) * a_stride); // [kStages][kRowTile] row norms
    float* c_nn = sN + kStages * kRowTile;                // [kColPairs] column norms
    int* c_lo = reinterpret_cast<int*>(c_nn + kColPairs); // [kColPairs] entry range [c_lo, c_hi)
    int* c_hi = c_lo + kColPairs;
    long long* c_off = reinterpret_cast<long long*>(c_hi + kColPairs); // [kColPairs] store offset of entry 0
    uint64_t* bars = reinterpret_cast<uint64_t*>(c_off + kColPairs);
    uint64_t* full = bars;              // [kStages]
    uint64_t* empty = bars + kStages;   // [kStages]
    uint64_t* tfull = bars + 2 * kStages; // [2]
    uint64_t* tempty = tfull + 2;       // [2]
    uint64_t* bfull = tempty + 2;       // [1]
    uint64_t* done = bfull + 1;         // [1]
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr uint32_t kCols = 2 * kColN;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1 + kEpiWarps);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(&tfull[s], 1);
            mbar_init(&tempty[s], kEpiWarps);
        }
        mbar_init(bfull, 1);
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < kColPairs) {
        const int n = n0 + int(threadIdx.x);
        int blo = 0, bhi = 0;
        long long off = 0;
        float nv = 0.f;
        if (n < nP) {
            blo = col_begin(n, capP);
            bhi = col_end(n, qP, nP);
            off = column_prefix(n, qP, nP, capP) - jb.kc_base - blo;
            nv = jb.nrm[n];
        }
        c_lo[threadIdx.x] = blo;
        c_hi[threadIdx.x] = bhi;
        c_off[threadIdx.x] = off;
        c_nn[threadIdx.x] = nv;
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
        // ---------------- producer: the column chunk once, then the band's row tiles ----------------
        if (lane == 0) {
            mbar_expect_tx(bfull, b_bytes);
            bulk_g2s(sB, jb.b_ops + size_t(ci) * b_bytes, b_bytes, bfull);
            int issued = 0;
            for (int i = 0; i < ntile; ++i) {
                const int s = i % kStages;
                if (i >= kStages && !mbar_wait(&empty[s], ((i / kStages) - 1) & 1, abort_flag, wait_ns)) break;
                ++issued;
                const int t = t0 + i;
                mbar_expect_tx(&full[s], a_bytes + kRowTile * 4);
                bulk_g2s(sA + size_t(s) * a_stride, jb.a_ops + size_t(t) * a_bytes, a_bytes, &full[s]);
                bulk_g2s(sN + s * kRowTile, jb.a_nrm + size_t(t) * kRowTile, kRowTile * 4, &full[s]);
            }
            mbar_drain(bfull, 0);
            for (int i = max(0, issued - kStages); i < issued; ++i) mbar_drain(&full[i % kStages], (i / kStages) & 1);
        }
    } else if (warp == kEpiWarps + 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0 && ntile > 0 && mbar_wait(bfull, 0, abort_flag, wait_ns)) {
            const uint32_t idesc = instr_desc<kMode>(kRowTile, kColN);
            const uint32_t lbo = 128 * 16; // both operands have 128 rows
            const int ksteps = jb.Kp / T::kStepK;
            const int lo_off = jb.Kp / T::kChunk;
            for (int i = 0; i < ntile; ++i) {
                const int s = i % kStages, buf = i & 1;
                if (!mbar_wait(&full[s], (i / kStages) & 1, abort_flag, wait_ns)) break;
                if (i >= 2 && !mbar_wait(&tempty[buf], ((i >> 1) - 1) & 1, abort_flag, wait_ns)) break;
                tc_fence_after();
                const uint8_t* a = sA + size_t(s) * a_stride;
                const uint32_t d = tmem + uint32_t(buf * kColN);
                for (int kk = 0; kk < ksteps; ++kk) {
                    const uint64_t ah = smem_desc(a + size_t(2 * kk) * lbo, lbo, 128);
                    const uint64_t bh = smem_desc(sB + size_t(2 * kk) * lbo, lbo, 128);
                    const uint64_t al = smem_desc(a + size_t(lo_off + 2 * kk) * lbo, lbo, 128);
                    const uint64_t bl = smem_desc(sB + size_t(lo_off + 2 * kk) * lbo, lbo, 128);
                    umma<kMode>(d, ah, bh, idesc, kk > 0 ? 1u : 0u);
                    umma<kMode>(d, ah, bl, idesc, 1u);
                    umma<kMode>(d, al, bh, idesc, 1u);
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
        // ---------------- epilogue: combined kernel values of the tile's band entries ----------------
        const int q = warp & 3, h = warp >> 2;
        const float ewl2 = jb.ewl2, wG = cm.wG, wL = cm.wL;
        float4* __restrict__ Kc = jb.Kc;
        for (int i = 0; i < ntile; ++i) {
            const int s = i % kStages, buf = i & 1;
            if (!mbar_wait(&full[s], (i / kStages) & 1, abort_flag, wait_ns)) break;
            if (!mbar_wait(&tfull[buf], (i >> 1) & 1, abort_flag, wait_ns)) break;
            tc_fence_after();
            const int b = (t0 + i) * kRowTile + q * 32 + lane; // this lane's row pair
            const float nb = sN[s * kRowTile + q * 32 + lane];
#pragma unroll 1
            for (int cb = 0; cb < kColN / 2; cb += 32) {
                const int col = h * (kColN / 2) + cb; // 32 accumulator columns = 16 column pairs
                float gv[32];
                tmem_ld32(tmem + (uint32_t(q * 32) << 16) + uint32_t(buf * kColN + col), gv);
#pragma unroll
                for (int jj = 0; jj < 16; ++jj) {
                    const int j = (col >> 1) + jj; // column pair within the chunk
                    if (b < c_lo[j] || b >= c_hi[j]) continue;
                    const float re = gv[2 * jj], im = -gv[2 * jj + 1];
                    const float sn = nb + c_nn[j];
                    const float A = wG * ex2(ewl2 * fmaxf(fmaf(-2.f, re, sn), 0.f));
                    const float Bp = wG * ex2(ewl2 * fmaxf(fmaf(-2.f, im, sn), 0.f));
                    const float Bm = wG * ex2(ewl2 * fmaxf(fmaf(2.f, im, sn), 0.f));
                    Kc[c_off[j] + b] = make_float4(fmaf(wL, re, A), fmaf(wL, im, Bp), fmaf(-wL, im, Bm), 0.f);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&tempty[buf]);
                mbar_arrive(&empty[s]);
            }
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

size_t kcol_tc_smem(int Kpmax)
{
    return op_bytes(kColN, Kpmax) + size_t(kStages) * op_bytes(kRowTile, Kpmax) + size_t(kStages) * kRowTile * 4 +
           size_t(kColPairs) * (4 + 4 + 4 + 8) + sizeof(uint64_t) * (2 * kStages + 6) + 16 + 1024;
}

} // namespace

int batch_kcol_tc_kp(int N) { return int(round_up(uint32_t(2 * N), uint32_t(tc::OpTraits<kMode>::kStepK))); }
int batch_kcol_tc_row_tile() { return kRowTile; }
int batch_kcol_tc_col_pairs() { return kColPairs; }
size_t batch_kcol_tc_a_bytes(int Kp) { return op_bytes(kRowTile, Kp); }
size_t batch_kcol_tc_b_bytes(int Kp) { return op_bytes(kColN, Kp); }

cudaError_t launch_batch_kcol_tc(const BatchKcolTcJob* d_jobs, int n_jobs, int max_units, const int* d_chunk_prefix,
                                 int total_chunks, int Kpmax, BatchCommon cm, int* d_err, cudaStream_t s)
{
    if (n_jobs <= 0) return cudaSuccess;
    if (Kpmax % tc::OpTraits<kMode>::kStepK != 0 || Kpmax > 64) return cudaErrorInvalidValue;
    if (max_units > 0) kcol_tc_pack_kernel<<<dim3(max_units, n_jobs), 256, 0, s>>>(d_jobs);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || total_chunks <= 0) return e;
    // every CTA holds 256 TMEM columns: at most two CTAs per SM (512 columns), so shared memory
    // is padded to more than a third of the SM's
    const size_t smem = std::max<size_t>(kcol_tc_smem(Kpmax), 80 * 1024);
    e = cudaFuncSetAttribute(kcol_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    kcol_tc_kernel<<<total_chunks, kThreads, smem, s>>>(d_jobs, n_jobs, d_chunk_prefix, Kpmax, cm, d_err,
                                                         wait_limit_ns());
    return cudaGetLastError();
}

} // namespace apsm
