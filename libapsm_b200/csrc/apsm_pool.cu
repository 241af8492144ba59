// Detector pool: resident state of many detectors and batched train/detect
// (the apsm_pool_* entry points of include/apsm_b200.h).
//
// A batch is laid out in one scratch buffer of its lane: the job descriptors
// (filled in a pinned host buffer, one copy), the staged host inputs, each
// training job's universe (its dictionary pairs, then the new pilots), kernel
// columns, and each detection job's packed samples.  Launch order
// on the lane's stream: dictionary -> universe copies, packing, kernel
// columns, the persistent sweep, universe tail -> dictionary copies, then the
// detection launches (one per antenna class).
#include "apsm_batch.cuh"
#include <cuda.h>
#include "apsm_host.hpp"
#include "apsm_tc.cuh"

#include <algorithm>
#include <array>
#include <atomic>
#include <condition_variable>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace apsm;

namespace {

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct PoolDet {
    bool live = false;
    uint32_t N = 0, Np = 0, cap = 0, capP = 0;
    uint32_t used = 0; // rows (2 per complex entry)
    float ew = 0.f;
    void* mem = nullptr;
    size_t bytes = 0;
    float2* Y = nullptr; // capP x Np dictionary pairs, oldest first
    float* nrm = nullptr;
    float* y = nullptr; // cap targets
    float* a = nullptr; // cap coefficients
    float* w = nullptr; // 2N
    float* r = nullptr; // 2N residual weights of the training sweep (w minus the dictionary's share)
};

struct Lane {
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[6] = {};     // train start/end, detect start/end, sweep start/end
    cudaEvent_t done = nullptr;                                // end of the last batch
    cudaEvent_t desc_copied = nullptr;                         // the pinned descriptors were consumed
    // detection inputs copied while the batch trains: a second stream, ordered after the
    // lane's earlier work (ev_start) and joined before each detection segment (seg_ev)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_start = nullptr;
    std::vector<cudaEvent_t> seg_ev; // per detection segment: its samples arrived
    // training samples packed on the copy stream, one launch per antenna class (the kernel
    // columns of a class wait for its pack only)
    cudaEvent_t ev_pack[5] = {};
    bool have_train = false, have_detect = false;
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    void* pinned = nullptr; // descriptors and staged host inputs of a batch (one H2D copy)
    size_t pinned_bytes = 0;
    void* pinned_out = nullptr; // estimates of a host-buffer batch (one D2H copy)
    size_t pinned_out_bytes = 0;
    struct CopyOut {
        void* dst;
        size_t off, bytes;
    };
    std::vector<CopyOut> pending; // estimates to hand to the caller once the batch finished
    std::vector<void*> retired;   // outgrown page-locked buffers (freed with the pool)
    int* err = nullptr;           // error flag of the last batch (in the scratch)
    int* err_host = nullptr;      // its copy in page-locked memory, written by the batch's last copy
    bool err_copied = false;      // the last batch copies the flag (it has kernels that can set it)
    bool unfinished = false;      // an APSM_RUN_HOST_ASYNC batch whose finish() has not run yet
    int launches = 0;             // kernels launched by the last batch
    // batch timeline (APSM_POOL_TRACE): stream start, inputs copied, packed, kernel columns, swept,
    // trained (dictionary copied back), detected
    cudaEvent_t tr[7] = {};
    cudaEvent_t tr_copy[2] = {}; // copy stream of a host-input batch: training samples packed, detection samples in
    bool tr_overlap = false;
    double t_run0 = 0, t_run1 = 0;
    double t_mark[3] = {0, 0, 0}; // run(): planned, descriptors written, inputs staged
    int tr_nT = 0, tr_nD = 0;
    bool traced = false;
};

double host_us()
{
    using namespace std::chrono;
    return duration<double, std::micro>(steady_clock::now().time_since_epoch()).count();
}

// Page-locked host memory (cudaMallocHost or cudaHostRegister): copies need no staging.
// A device address for the bytes [p, p + bytes) when they lie inside one page-locked host
// allocation mapped for the device (kernels then read them over the bus); nullptr otherwise.
const void* device_view(const void* p, size_t bytes)
{
    if (!p || bytes == 0) return nullptr;
    // the driver's pointer query (all four attributes in one call; a batch asks for every
    // input and output buffer), looked up through the runtime (the library links no libcuda)
    using PtrAttrsFn = CUresult (*)(unsigned int, CUpointer_attribute*, void**, CUdeviceptr);
    static PtrAttrsFn cuPointerGetAttributes = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuPointerGetAttributes", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            fn = nullptr;
        }
        return reinterpret_cast<PtrAttrsFn>(fn);
    }();
    if (!cuPointerGetAttributes) return nullptr;
    const CUdeviceptr a = CUdeviceptr(reinterpret_cast<uintptr_t>(p));
    unsigned int type = 0;
    CUdeviceptr start = 0, dptr = 0;
    size_t size = 0;
    CUpointer_attribute attrs[4] = {CU_POINTER_ATTRIBUTE_MEMORY_TYPE, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR,
                                    CU_POINTER_ATTRIBUTE_RANGE_SIZE, CU_POINTER_ATTRIBUTE_DEVICE_POINTER};
    void* data[4] = {&type, &start, &size, &dptr};
    // (memory the driver does not know reads as type 0: not page-locked)
    if (cuPointerGetAttributes(4, attrs, data, a) != CUDA_SUCCESS || type != CU_MEMORYTYPE_HOST) return nullptr;
    if (a < start || a - start > size || bytes > size - (a - start) || dptr == 0) return nullptr;
    return reinterpret_cast<const void*>(dptr);
}

bool is_pinned(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Copies host inputs into a lane's page-locked staging buffer.  Batches of more
// than kStageSplit bytes are cut into byte ranges shared with persistent helper
// threads (started on first use), so a request loop does not pay for thread
// creation and a large batch is not staged at one thread's memcpy bandwidth.
class Stager {
public:
    ~Stager()
    {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }

    struct Range {
        char* dst;
        const char* src;
        size_t bytes;
    };

    void copy(const std::vector<Range>& pieces)
    {
        begin(pieces);
        wait();
    }

    // Starts the copies (small totals: done here and now) and returns; wait() joins them,
    // the calling thread taking pieces too.
    void begin(const std::vector<Range>& pieces)
    {
        wait();
        size_t total = 0;
        for (const auto& r : pieces) total += r.bytes;
        if (total < kStageSplit) {
            for (const auto& r : pieces) std::memcpy(r.dst, r.src, r.bytes);
            return;
        }
        start();
        // cut every input into kStageGrain pieces; helpers and the waiting thread take pieces in turn
        work_own_.clear();
        for (const auto& r : pieces)
            for (size_t o = 0; o < r.bytes; o += kStageGrain)
                work_own_.push_back({r.dst + o, r.src + o, std::min(kStageGrain, r.bytes - o)});
        // one helper per kPiecesPerHelper pieces at most: a request-sized batch wakes a few
        // helpers, not every core (which would preempt the threads serving requests)
        const unsigned want = unsigned(std::min(th_.size(), work_own_.size() / kPiecesPerHelper));
        {
            std::lock_guard<std::mutex> g(mu_);
            work_ = &work_own_;
            next_.store(0);
            busy_ = want;
            want_ = want;
            ++gen_;
        }
        active_ = true;
        if (want > 0) cv_.notify_all();
    }

    void wait()
    {
        if (!active_) return;
        drain(work_own_);
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return busy_ == 0; });
        work_ = nullptr;
        active_ = false;
    }

private:
    static constexpr size_t kStageSplit = size_t(1) << 20;
    static constexpr size_t kStageGrain = size_t(256) << 10;
    static constexpr size_t kPiecesPerHelper = 8;

    void drain(std::vector<Range>& work)
    {
        for (size_t i = next_.fetch_add(1); i < work.size(); i = next_.fetch_add(1))
            std::memcpy(work[i].dst, work[i].src, work[i].bytes);
    }

    void start()
    {
        if (!th_.empty()) return;
        const unsigned hw = std::thread::hardware_concurrency();
        const unsigned n = std::min(15u, std::max(1u, hw > 1 ? hw - 1 : 1u));
        for (unsigned k = 0; k < n; ++k)
            th_.emplace_back([this, k] {
                uint64_t seen = 0;
                for (;;) {
                    std::vector<Range>* w;
                    {
                        std::unique_lock<std::mutex> lk(mu_);
                        cv_.wait(lk, [&] { return stop_ || (gen_ != seen && k < want_); });
                        if (stop_) return;
                        seen = gen_;
                        w = work_;
                    }
                    drain(*w);
                    std::lock_guard<std::mutex> g(mu_);
                    if (--busy_ == 0) done_cv_.notify_all();
                }
            });
    }

    std::vector<std::thread> th_;
    std::vector<Range> work_own_; // pieces of the copies in flight
    bool active_ = false;         // begin() started copies that wait() has not joined
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    std::vector<Range>* work_ = nullptr;
    std::atomic<size_t> next_{0};
    unsigned busy_ = 0;
    unsigned want_ = 0; // helpers taking part in the current copies
    uint64_t gen_ = 0;
    bool stop_ = false;
};

constexpr size_t kDirectOutJobs = 16; // detection jobs whose estimates are copied to the caller one by one
constexpr size_t kZeroCopyMin = size_t(4) << 20; // training inputs read in place from this many bytes on
constexpr size_t kSplitGroup = size_t(32) << 20;  // pageable detection samples staged and uploaded in groups of this size
constexpr size_t kArenaJobs = 32;     // training jobs from which a batch reads its step lists from the arena

int detect_class(uint32_t N)
{
    for (int c : {4, 8, 16, 32, 64})
        if (int(N) <= c) return c;
    return 0;
}

} // namespace

struct apsm_pool {
    Config cfg;
    int gram_mode = kTF32x3; // GramMode of tensor-core detection (cfg.detect_mode != Exact)
    BatchCommon cm{};
    uint64_t budget = 0;
    uint64_t resident = 0;
    std::vector<PoolDet> dets;
    std::vector<Lane> lanes;
    int device = 0, sms = 0, sweep_ctas = 1;
    // launch shapes (0: the built-in choice), set by apsm_pool_autotune
    struct Shape {
        int sweep_per_sm = 0;         // training-sweep CTAs per SM (1 .. sweep_ctas)
        int gram_stages = 0;          // tensor-core detection: dictionary chunks in flight (2, 3)
        int detect_blocks_per_sm = 0; // CUDA-core detection: blocks per SM below which chunks are split
    } shape;
    std::string last_error;
    std::mutex mu;
    std::FILE* trace = nullptr; // batch timeline lines (env APSM_POOL_TRACE = file path)
    bool timing = true;         // per-stage GPU events of each batch (apsm_pool_last_ms)
    uint32_t fault_lane_alloc = 0; // lane-scratch growths still to fail (apsm_pool_inject_fault)
    // Form of the kernel columns of a training job, decided by the job alone (so a job's result
    // never depends on its batch): tensor cores for fresh sweeps (no old-pair sums) with
    // kcol_tc_min_n <= N <= 32 antennas, the CUDA-core kernel otherwise.  APSM_POOL_KCOL=cuda
    // or =tensor (read at creation) forces one form where it applies.
    int kcol_tc_min_n = 8;
    bool kcol_tc_off = false;
    // normConstraint > 0: training jobs run the single detector's exact sweep, which applies the
    // constraint after every step (apsm_train.cu:142-145, 168-256); one such detector per antenna
    // count, created on first use, holds a pool detector's state while it trains
    std::map<uint32_t, apsm_detector*> exact_by_n;
    apsm_status exact_handle(uint32_t N, apsm_detector** out);
    apsm_status train_exact(uint32_t lane, const apsm_job* jobs, uint32_t n, int mode, std::vector<apsm_job>* rest);
    cudaMemPool_t mempool = nullptr; // lane scratch (stream-ordered; keeps its memory mapped)
    Stager stager;                   // host-input staging (helper threads for large batches)
    std::map<uint32_t, std::vector<int>> perms;
    // training schedules by (rows before the call, pilots): the same request shapes recur
    // from batch to batch, and a batch of 512 detectors would rebuild ~600 k steps each time
    struct Schedule {
        std::vector<TrainStep> steps;
        int final_hi = 0;
        long long dev = -1; // offset of its copy in sched_arena (-1: none)
    };
    std::map<std::pair<uint32_t, uint32_t>, Schedule> schedules;
    Schedule& schedule(uint32_t used_before, uint32_t P)
    {
        auto it = schedules.find({used_before, P});
        if (it == schedules.end()) {
            Schedule sc;
            sc.steps = build_schedule(cfg, used_before, P, 2 * cfg.dict_size, &sc.final_hi);
            it = schedules.emplace(std::make_pair(used_before, P), std::move(sc)).first;
        }
        return it->second;
    }
    // Device copies of the schedules for batches of many training jobs, so such a batch
    // uploads (and stages) no step lists once their shapes recur: one arena, each schedule
    // uploaded (synchronously) the first time a large batch uses it; reset, with every lane
    // idle, when full.  Small batches carry their few steps in the descriptor upload.
    DevBuf<TrainStep> sched_arena;
    size_t sched_used = 0;
    cudaStream_t sched_stream = nullptr;

    ~apsm_pool();
    apsm_status fail(apsm_status st, const std::string& msg)
    {
        last_error = msg;
        return st;
    }
    apsm_status cuda_fail(cudaError_t e, const char* what)
    {
        cudaGetLastError();
        last_error = std::string(what) + ": " + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? APSM_ERR_OUT_OF_MEMORY : APSM_ERR_CUDA;
    }
    uint64_t in_use() const
    {
        uint64_t s = resident + sizeof(TrainStep) * sched_arena.n;
        for (const auto& l : lanes) s += l.scratch_bytes;
        return s;
    }
    size_t train_bytes(const PoolDet& d, uint32_t P, bool host) const;
    size_t detect_bytes(const PoolDet& d, uint32_t S, bool host) const;
    // reserve_only: plan the batch and grow the lane's buffers to its needs, run nothing
    apsm_status run(uint32_t lane, const apsm_job* jobs, uint32_t n, int mode, bool reserve_only = false);
    apsm_status check_lane(uint32_t lane);
    // Checks of one job that need no other job of its batch (touches no pool state).
    apsm_status job_error(const apsm_job& j, std::string* msg) const
    {
        if (j.detector >= dets.size() || !dets[j.detector].live) {
            *msg = "unknown detector";
            return APSM_ERR_INVALID_ARGUMENT;
        }
        if (j.kind != APSM_JOB_TRAIN && j.kind != APSM_JOB_DETECT) {
            *msg = "unknown kind";
            return APSM_ERR_INVALID_ARGUMENT;
        }
        if (j.length == 0) return APSM_OK;
        if (!j.rx) *msg = "null rx";
        else if (j.kind == APSM_JOB_TRAIN && !j.tx) *msg = "null tx";
        else if (j.kind == APSM_JOB_DETECT && !j.est) *msg = "null est";
        else return APSM_OK;
        return APSM_ERR_INVALID_ARGUMENT;
    }
    apsm_status check_job(const apsm_job& j, const std::string& what)
    {
        std::string msg;
        const apsm_status st = job_error(j, &msg);
        return st == APSM_OK ? st : fail(st, what + ": " + msg);
    }
    apsm_status finish(uint32_t lane); // wait for the lane, hand out estimates, check its error flag
    apsm_status autotune(uint32_t lane, const apsm_job* jobs, uint32_t n, int mode, std::string* report);
};

#define POOL_CK(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) return p->cuda_fail(e_, #call);                         \
    } while (0)

apsm_pool::~apsm_pool()
{
    for (auto& kv : exact_by_n) delete kv.second;
    for (auto& l : lanes) {
        if (l.stream) cudaStreamSynchronize(l.stream);
        if (l.scratch) cudaFree(l.scratch);
        if (l.pinned) cudaFreeHost(l.pinned);
        if (l.pinned_out) cudaFreeHost(l.pinned_out);
        for (void* r : l.retired) cudaFreeHost(r);
        for (auto& e : l.ev)
            if (e) cudaEventDestroy(e);
        if (l.done) cudaEventDestroy(l.done);
        if (l.desc_copied) cudaEventDestroy(l.desc_copied);
        if (l.copy_stream) cudaStreamSynchronize(l.copy_stream);
        if (l.ev_start) cudaEventDestroy(l.ev_start);
        for (auto& e : l.ev_pack)
            if (e) cudaEventDestroy(e);
        for (auto& e : l.seg_ev)
            if (e) cudaEventDestroy(e);
        if (l.copy_stream) cudaStreamDestroy(l.copy_stream);
        for (auto& e : l.tr)
            if (e) cudaEventDestroy(e);
        for (auto& e : l.tr_copy)
            if (e) cudaEventDestroy(e);
        if (l.err_host) cudaFreeHost(l.err_host);
        if (l.stream) cudaStreamDestroy(l.stream);
    }
    if (sched_stream) {
        cudaStreamSynchronize(sched_stream);
        cudaStreamDestroy(sched_stream);
    }
    for (auto& d : dets)
        if (d.mem) cudaFree(d.mem);
    if (mempool) cudaMemPoolDestroy(mempool);
    if (trace) std::fclose(trace);
}

namespace {

// Bytes of a detector's resident state and its sub-buffer offsets.
size_t resident_layout(uint32_t N, uint32_t capP, size_t off[6])
{
    const uint32_t Np = round_up(N, 2);
    size_t o = 0;
    off[0] = o; o = align_up(o + sizeof(float2) * size_t(capP) * Np, 256);
    off[1] = o; o = align_up(o + sizeof(float) * capP, 256);
    off[2] = o; o = align_up(o + sizeof(float) * 2 * capP, 256);
    off[3] = o; o = align_up(o + sizeof(float) * 2 * capP, 256);
    off[4] = o; o = align_up(o + sizeof(float) * 2 * N, 256);
    off[5] = o; o = align_up(o + sizeof(float) * 2 * N, 256);
    return o;
}

struct TrainPlan {
    uint32_t job = 0; // index in the caller's list
    PoolDet* det = nullptr;
    const std::vector<TrainStep>* steps = nullptr; // the pool's cached schedule for (rows before, P)
    const void* zc_rx = nullptr; // host-buffer batch: the caller's pilots as the device reads them in place
    const void* zc_tx = nullptr;
    long long* steps_dev = nullptr; // its offset in the pool's device schedule arena (-1: not there)
    int final_hi = 0;
    uint32_t P = 0, usedP = 0, nP = 0, n_first = 0;
    long long kc_base = 0, n_kc = 0;
    size_t off_rx = 0, off_tx = 0, off_Y = 0, off_nrm = 0, off_y = 0, off_a = 0, off_kc = 0;
    size_t off_steps = 0;
    uint32_t usedP_new = 0, lo_new = 0;
    const int* perm_dev = nullptr;
    size_t perm_off = 0;
    bool fresh = false;
    // prologue sums of the first window's pairs over the old pairs (launch_batch_kcol)
    int pro_n = 0, pro_w = 0, pro_lo = 0, pro_stride = 0; // pro_n: columns with sums
    size_t off_pro = 0;
    // kernel columns on the tensor cores (launch_batch_kcol_tc): operand scratch
    bool kc_tc = false;
    int kc_Kp = 0, kc_a_tiles = 0, kc_b_chunks = 0;
    size_t off_kca = 0, off_kcb = 0, off_kcn = 0;
};

struct DetectPlan {
    uint32_t job = 0;
    PoolDet* det = nullptr;
    uint32_t S = 0, Mp = 0;
    int cls = 0;       // CUDA-core class (max antennas) or tensor-core class (max Kp)
    bool gram = false; // tensor-core (tcgen05) form
    int Kp = 0, tiles = 0, chunks = 0;
    size_t off_rx = 0, off_Y = 0, off_nrm = 0, off_est = 0;
    void* zc_est = nullptr; // host-buffer batch: the caller's estimates as the device writes them in place
    size_t off_aops = 0, off_bops = 0, off_bx = 0, off_lin = 0;
    size_t off_part = 0, off_cnt = 0; // split CUDA-core launches: chunk sums, tile counters
};

int gram_class(int Kp)
{
    for (int c : {8, 16, 32, 64})
        if (Kp <= c) return c;
    return 0;
}

} // namespace

size_t apsm_pool::train_bytes(const PoolDet& d, uint32_t P, bool host) const
{
    const size_t usedP = d.used / 2, nP = usedP + P;
    const size_t q = size_t(cm.qP);
    size_t b = 0;
    if (host) b += align_up(sizeof(float2) * d.N * P, 256) + align_up(sizeof(float2) * P, 256);
    b += align_up(sizeof(float2) * nP * d.Np, 256) + align_up(sizeof(float) * nP, 256) +
         2 * align_up(sizeof(float) * 2 * nP, 256);
    // kernel columns: at most min(capP, nP) + q entries per pair of the first window onwards
    const size_t first = usedP > q ? usedP - q : 0;
    const size_t cols = nP - first;
    const size_t len = std::min<size_t>(d.capP, nP) + q;
    b += align_up(sizeof(float4) * cols * len, 256);
    b += align_up(sizeof(TrainStep) * (size_t(cfg.passes) * (P + q + 2) + 4), 256) + align_up(sizeof(int) * P, 256);
    b += 4 * sizeof(BatchTrainJob) + 4 * sizeof(BatchPackJob) + 4 * sizeof(BatchCopyJob);
    return b;
}

size_t apsm_pool::detect_bytes(const PoolDet& d, uint32_t S, bool host) const
{
    size_t b = align_up(sizeof(float2) * size_t(S) * d.Np, 256) + align_up(sizeof(float) * S, 256);
    if (host) b += align_up(sizeof(float2) * size_t(d.N) * S, 256) + align_up(sizeof(float2) * S, 256);
    return b + sizeof(BatchDetectJob) + sizeof(BatchPackJob);
}

apsm_status apsm_pool::run(uint32_t lane_id, const apsm_job* jobs, uint32_t n, int mode, bool reserve_only)
{
    apsm_pool* p = this;
    Lane& L = lanes[lane_id];
    const bool host = mode != APSM_RUN_DEVICE;
    const double t_run0 = trace ? host_us() : 0.0;
    if (!L.pending.empty() || L.unfinished) {
        apsm_status st = finish(lane_id); // the lane's previous host batch (its estimates, its error flag)
        if (st != APSM_OK) return st;
    }
    const uint32_t cap = 2 * cfg.dict_size;
    if (schedules.size() > 16384) schedules.clear(); // bounded; no plan holds a pointer between batches

    // ---------- validate ----------
    std::vector<char> trained(dets.size(), 0);
    for (uint32_t i = 0; i < n; ++i) {
        const apsm_job& j = jobs[i];
        const apsm_status st = check_job(j, "job " + std::to_string(i));
        if (st != APSM_OK) return st;
        if (j.kind == APSM_JOB_TRAIN && (j.length > 0 || (j.flags & APSM_JOB_FRESH))) {
            if (trained[j.detector])
                return fail(APSM_ERR_INVALID_ARGUMENT, "detector " + std::to_string(j.detector) +
                                                           " is trained twice in one batch");
            trained[j.detector] = 1;
        }
    }

    // normConstraint: the training jobs first, each with the exact sweep; the batch then holds the
    // detection jobs (which see this training, as in every batch)
    std::vector<apsm_job> rest;
    if (cfg.norm_constraint > 0.f && !reserve_only) {
        const apsm_status st = train_exact(lane_id, jobs, n, mode, &rest);
        if (st != APSM_OK) return st;
        jobs = rest.data();
        n = uint32_t(rest.size());
    }

    // ---------- plan (sizes and offsets) ----------
    std::vector<TrainPlan> tp;
    std::vector<DetectPlan> dp;
    for (uint32_t i = 0; i < n; ++i)
        if (jobs[i].kind == APSM_JOB_TRAIN && jobs[i].length > 0) {
            TrainPlan t;
            t.job = i;
            t.det = &dets[jobs[i].detector];
            t.P = jobs[i].length;
            t.fresh = (jobs[i].flags & APSM_JOB_FRESH) != 0;
            const uint32_t used0 = t.fresh ? 0u : t.det->used;
            Schedule& sc = schedule(used0, t.P);
            t.steps = &sc.steps;
            t.steps_dev = &sc.dev;
            t.final_hi = sc.final_hi;
            t.usedP = used0 / 2;
            t.nP = t.usedP + t.P;
            t.n_first = t.steps->empty() ? t.nP : uint32_t((*t.steps)[0].hi - (*t.steps)[0].wk) / 2;
            t.kc_base = column_prefix(t.n_first, cm.qP, t.nP, t.det->capP);
            t.n_kc = column_prefix(t.nP, cm.qP, t.nP, t.det->capP) - t.kc_base;
            if (!t.steps->empty() && t.usedP > 0 && !t.fresh) {
                const int hiP0 = (*t.steps)[0].hi / 2;
                t.pro_w = hiP0 - int(t.n_first);
                t.pro_n = int(t.nP - t.n_first);
                t.pro_lo = std::max(0, hiP0 - int(t.det->capP));
                t.pro_stride = (int(t.det->capP) + cm.qP + kKcolGroup - 2 + kKcolRows - 1) / kKcolRows + 1;
            }
            const uint32_t fhP = uint32_t(t.final_hi) / 2;
            t.usedP_new = std::min(fhP, t.det->capP);
            t.lo_new = fhP - t.usedP_new;
            t.kc_tc = !kcol_tc_off && t.pro_n == 0 && t.nP > t.n_first && int(t.det->N) >= kcol_tc_min_n &&
                      t.det->N <= 32;
            if (t.kc_tc) {
                t.kc_Kp = batch_kcol_tc_kp(int(t.det->N));
                t.kc_a_tiles = int((t.nP + batch_kcol_tc_row_tile() - 1) / batch_kcol_tc_row_tile());
                t.kc_b_chunks = int((t.nP - t.n_first + batch_kcol_tc_col_pairs() - 1) / batch_kcol_tc_col_pairs());
            }
            tp.push_back(std::move(t));
        }
    // step lists of a large batch from the device arena (new ones uploaded now)
    const bool arena = tp.size() >= kArenaJobs;
    if (arena) {
        size_t fresh_steps = 0, all_steps = 0;
        for (const auto& t : tp) {
            all_steps += t.steps->size();
            if (*t.steps_dev < 0) fresh_steps += t.steps->size();
        }
        if (sched_used + fresh_steps > sched_arena.n) {
            // full: every lane idle, then start over (and grow to hold at least this batch)
            for (auto& l : lanes) {
                POOL_CK(cudaStreamSynchronize(l.stream));
                POOL_CK(cudaStreamSynchronize(l.copy_stream));
            }
            for (auto& kv : schedules) kv.second.dev = -1;
            sched_used = 0;
            if (all_steps > sched_arena.n) {
                const size_t want = std::max(all_steps + all_steps / 2, size_t(1) << 20);
                const uint64_t others = in_use() - sizeof(TrainStep) * sched_arena.n;
                if (budget && others + sizeof(TrainStep) * want > budget)
                    return fail(APSM_ERR_OUT_OF_MEMORY, "the batch's training schedules exceed the HBM budget");
                POOL_CK(sched_arena.ensure(want));
            }
        }
        for (auto& t : tp)
            if (*t.steps_dev < 0) {
                *t.steps_dev = (long long)sched_used;
                POOL_CK(cudaMemcpyAsync(sched_arena.p + sched_used, t.steps->data(), sizeof(TrainStep) * t.steps->size(),
                                        cudaMemcpyHostToDevice, sched_stream));
                sched_used += t.steps->size();
            }
        POOL_CK(cudaStreamSynchronize(sched_stream)); // in place before any lane's later batch reads it
    }
    // longest sweeps first (the persistent kernel takes jobs in this order)
    std::stable_sort(tp.begin(), tp.end(),
                     [](const TrainPlan& x, const TrainPlan& y) { return x.steps->size() > y.steps->size(); });
    // dictionary sizes after this batch's training, for the detection jobs
    std::vector<uint32_t> used_after(dets.size());
    for (size_t d = 0; d < dets.size(); ++d) used_after[d] = dets[d].used;
    std::vector<PoolDet*> resets;
    for (uint32_t i = 0; i < n; ++i)
        if (jobs[i].kind == APSM_JOB_TRAIN && jobs[i].length == 0 && (jobs[i].flags & APSM_JOB_FRESH)) {
            resets.push_back(&dets[jobs[i].detector]);
            used_after[jobs[i].detector] = 0;
        }
    for (const auto& t : tp) used_after[jobs[t.job].detector] = 2 * t.usedP_new;
    for (uint32_t i = 0; i < n; ++i)
        if (jobs[i].kind == APSM_JOB_DETECT && jobs[i].length > 0) {
            DetectPlan d;
            d.job = i;
            d.det = &dets[jobs[i].detector];
            d.S = jobs[i].length;
            d.Mp = used_after[jobs[i].detector] / 2;
            d.gram = cfg.detect_mode != DetectMode::Exact && d.det->N <= 32;
            if (d.gram) {
                d.Kp = batch_gram_kp(gram_mode, int(d.det->N));
                d.cls = gram_class(d.Kp);
                d.tiles = int((d.S + batch_gram_tile() - 1) / batch_gram_tile());
                const int cp = batch_gram_chunk_pairs(gram_mode, d.Kp);
                d.chunks = int((d.Mp + cp - 1) / cp);
            } else {
                d.cls = detect_class(d.det->N);
            }
            dp.push_back(d);
        }
    std::stable_sort(dp.begin(), dp.end(), [](const DetectPlan& x, const DetectPlan& y) {
        return x.gram != y.gram ? x.gram < y.gram : x.cls < y.cls;
    });
    size_t nG = 0, nGcls = 0;
    for (size_t k = 0; k < dp.size(); ++k)
        if (dp[k].gram) {
            ++nG;
            if (k == 0 || !dp[k - 1].gram || dp[k - 1].cls != dp[k].cls) ++nGcls;
        }

    const size_t nT = tp.size(), nD = dp.size();
    // CUDA-core detection: when the batch's sample tiles alone would leave most of the GPU idle
    // (single requests), the dictionary chunks of each tile are spread over several blocks;
    // the estimates do not depend on this (launch_batch_detect)
    int det_parts = 1;
    {
        long long tiles_all = 0;
        int chunks_max = 0;
        const int tile = batch_detect_tile(), chunk = batch_detect_chunk();
        for (size_t k = 0; k < nD - nG; ++k) {
            tiles_all += (dp[k].S + tile - 1) / tile;
            chunks_max = std::max(chunks_max, int((dp[k].Mp + chunk - 1) / chunk));
        }
        const long long target = (shape.detect_blocks_per_sm > 0 ? shape.detect_blocks_per_sm : 4LL) * std::max(1, sms);
        if (tiles_all > 0 && tiles_all < target)
            det_parts = int(std::min<long long>(std::max(chunks_max, 1), (target + tiles_all - 1) / tiles_all));
    }
    size_t nCopyIn = 0;
    for (const auto& t : tp) nCopyIn += t.usedP > 0;
    const size_t nPack = nT; // detection reads the samples as the caller holds them
    // Training inputs of a large host-buffer batch in page-locked, device-mapped buffers are
    // read in place by the packing kernel (no staging copy, no upload); small batches stage
    // them (a copy of a few KB costs less than reading them over the bus).
    bool zc_train = false;
    if (host && nT > 0) {
        size_t bytes = 0;
        for (const auto& t : tp) bytes += sizeof(float2) * (size_t(t.det->N) + 1) * t.P;
        zc_train = bytes >= kZeroCopyMin;
        for (auto& t : tp) {
            if (!zc_train) break;
            const apsm_job& j = jobs[t.job];
            t.zc_rx = device_view(j.rx, sizeof(float2) * size_t(t.det->N) * t.P);
            t.zc_tx = device_view(j.tx, sizeof(float2) * t.P);
            zc_train = t.zc_rx && t.zc_tx;
        }
    }
    // Estimates of a large host-buffer batch into page-locked, device-mapped buffers are written
    // there by the detection kernels (no copy back, no scatter).
    bool zc_est = false;
    if (host && nD > 0) {
        size_t bytes = 0;
        for (const auto& q : dp) bytes += sizeof(float2) * q.S;
        zc_est = bytes >= kZeroCopyMin;
        for (auto& q : dp) {
            if (!zc_est) break;
            q.zc_est = const_cast<void*>(device_view(jobs[q.job].est, sizeof(float2) * q.S));
            zc_est = q.zc_est != nullptr;
        }
    }
    // descriptor region
    size_t o = 0;
    const size_t off_tj = o; o = align_up(o + sizeof(BatchTrainJob) * nT, 256);
    const size_t off_dj = o; o = align_up(o + sizeof(BatchDetectJob) * nD, 256);
    const size_t off_pj = o; o = align_up(o + sizeof(BatchPackJob) * nPack, 256);
    const size_t off_ci = o; o = align_up(o + sizeof(BatchCopyJob) * nCopyIn, 256);
    const size_t off_co = o; o = align_up(o + sizeof(BatchCopyJob) * nT, 256);
    const size_t off_ko = o; o = align_up(o + sizeof(int) * nT, 256); // training jobs by antenna class
    const size_t off_kt = o; o = align_up(o + sizeof(BatchKcolTcJob) * nT, 256); // tensor-core column jobs
    const size_t off_ktp = o; o = align_up(o + sizeof(int) * (nT + 5), 256);     // their chunk prefixes
    const size_t off_gj = o; o = align_up(o + sizeof(BatchGramJob) * nG, 256);
    const size_t off_gp = o; o = align_up(o + sizeof(int) * (nG + nGcls), 256);
    if (!arena)
        for (auto& t : tp) {
            t.off_steps = o;
            o = align_up(o + sizeof(TrainStep) * t.steps->size(), 16);
        }
    std::map<uint32_t, size_t> perm_off;
    if (cfg.shuffle)
        for (auto& t : tp) {
            if (!perm_off.count(t.P)) {
                perm_off[t.P] = o;
                o = align_up(o + sizeof(int) * t.P, 16);
                if (!perms.count(t.P)) perms[t.P] = shuffle_permutation(t.P);
            }
            t.perm_off = perm_off[t.P];
        }
    o = align_up(o, 256);
    // sweep job counter + error flag, and the tile counters of split CUDA-core detection: zeroed
    // in the host copy of the descriptors, so the one upload clears them
    const size_t off_counter = o;
    o = align_up(o + 256, 256);
    const size_t off_dcnt = o;
    if (det_parts > 1)
        for (auto& d : dp)
            if (!d.gram) {
                d.off_cnt = o;
                o += sizeof(int) * ((d.S + batch_detect_tile() - 1) / batch_detect_tile());
            }
    o = align_up(o, 256);
    const size_t dcnt_bytes = o - off_dcnt;
    if (host) { // staged host inputs travel with the descriptors
        if (!zc_train)
            for (auto& t : tp) {
                t.off_rx = o; o = align_up(o + sizeof(float2) * size_t(t.det->N) * t.P, 16);
                t.off_tx = o; o = align_up(o + sizeof(float2) * t.P, 16);
            }
        for (auto& d : dp) {
            d.off_rx = o;
            o = align_up(o + sizeof(float2) * size_t(d.det->N) * d.S, 16);
        }
        o = align_up(o, 256);
    }
    const size_t desc_bytes = o; // bytes of the one host-to-device copy
    const size_t off_det_in = host && nD > 0 ? dp[0].off_rx : desc_bytes; // detection samples from here
    for (auto& t : tp) {
        const PoolDet& d = *t.det;
        t.off_Y = o; o = align_up(o + sizeof(float2) * size_t(t.nP) * d.Np, 256);
        t.off_nrm = o; o = align_up(o + sizeof(float) * t.nP, 256);
        t.off_y = o; o = align_up(o + sizeof(float) * 2 * t.nP, 256);
        t.off_a = o; o = align_up(o + sizeof(float) * 2 * t.nP, 256);
        t.off_kc = o; o = align_up(o + sizeof(float4) * size_t(std::max<long long>(t.n_kc, 1)), 256);
        if (t.kc_tc) {
            t.off_kca = o; o = align_up(o + batch_kcol_tc_a_bytes(t.kc_Kp) * t.kc_a_tiles, 256);
            t.off_kcb = o; o = align_up(o + batch_kcol_tc_b_bytes(t.kc_Kp) * t.kc_b_chunks, 256);
            t.off_kcn = o; o = align_up(o + sizeof(float) * batch_kcol_tc_row_tile() * t.kc_a_tiles, 256);
        }
        if (t.pro_n > 0) {
            t.off_pro = o;
            o = align_up(o + sizeof(float2) * size_t(t.pro_n) * t.pro_stride, 256);
        }
    }
    for (auto& d : dp) {
        if (d.gram) {
            d.off_nrm = o; o = align_up(o + sizeof(float) * d.S, 256);
        }
        if (det_parts > 1 && !d.gram) {
            const size_t chunks = (d.Mp + batch_detect_chunk() - 1) / batch_detect_chunk();
            d.off_part = o;
            o = align_up(o + sizeof(float2) * size_t(d.S) * std::max<size_t>(chunks, 1), 256);
        }
        if (d.gram) {
            d.off_aops = o; o = align_up(o + batch_gram_a_bytes(gram_mode, d.Kp) * d.tiles, 256);
            d.off_bops = o; o = align_up(o + batch_gram_b_bytes(gram_mode, d.Kp) * std::max(d.chunks, 1), 256);
            d.off_bx = o; o = align_up(o + sizeof(float) * batch_gram_bx_floats(gram_mode, d.Kp) * std::max(d.chunks, 1), 256);
            d.off_lin = o; o = align_up(o + sizeof(float2) * d.S, 256);
        }
    }
    const size_t est_begin = o;
    if (host && !zc_est)
        for (auto& d : dp) {
            d.off_est = o;
            o = align_up(o + sizeof(float2) * d.S, 16);
        }
    const size_t est_bytes = o - est_begin;
    o = align_up(o, 256);
    const size_t scratch_need = o;

    const double t_plan = trace ? host_us() : 0.0;
    // ---------- memory ----------
    // Growth is geometric and never stalls the device: scratch comes from the pool's own
    // stream-ordered memory pool (the old block is released in stream order behind the lane's
    // earlier batches), and outgrown page-locked buffers are kept until the pool is destroyed
    // (freeing page-locked memory can synchronize the device).
    if (scratch_need > L.scratch_bytes) {
        const uint64_t others = in_use() - L.scratch_bytes;
        if (budget && others + scratch_need > budget)
            return fail(APSM_ERR_OUT_OF_MEMORY, "batch needs " + std::to_string(scratch_need) +
                                                    " scratch bytes; the HBM budget leaves " +
                                                    std::to_string(budget > others ? budget - others : 0));
        size_t want = std::max(scratch_need, 2 * L.scratch_bytes);
        if (budget && others + want > budget) want = size_t(budget - others);
        if (L.scratch) POOL_CK(cudaFreeAsync(L.scratch, L.stream));
        L.scratch = nullptr;
        L.scratch_bytes = 0;
        if (fault_lane_alloc > 0) { // injected (tests): this growth fails as an allocation would
            --fault_lane_alloc;
            return fail(APSM_ERR_OUT_OF_MEMORY, "lane scratch growth failed (injected fault)");
        }
        POOL_CK(cudaMallocFromPoolAsync(&L.scratch, want, mempool, L.stream));
        L.scratch_bytes = want;
    }
    if (desc_bytes > L.pinned_bytes) {
        POOL_CK(cudaEventSynchronize(L.desc_copied));
        if (L.pinned) L.retired.push_back(L.pinned);
        L.pinned = nullptr;
        const size_t want = std::max({desc_bytes + desc_bytes / 2, 2 * L.pinned_bytes, size_t(1) << 20});
        L.pinned_bytes = 0;
        POOL_CK(cudaMallocHost(&L.pinned, want));
        L.pinned_bytes = want;
    }
    if (est_bytes > L.pinned_out_bytes) {
        if (L.pinned_out) L.retired.push_back(L.pinned_out); // no batch of this lane has results pending
        L.pinned_out = nullptr;
        const size_t want = std::max({est_bytes + est_bytes / 2, 2 * L.pinned_out_bytes, size_t(1) << 18});
        L.pinned_out_bytes = 0;
        POOL_CK(cudaMallocHost(&L.pinned_out, want));
        L.pinned_out_bytes = want;
    }
    if (reserve_only) {
        POOL_CK(cudaStreamSynchronize(L.stream)); // the scratch is mapped now, not under a later batch
        return APSM_OK;
    }
    POOL_CK(cudaEventSynchronize(L.desc_copied)); // the previous batch's descriptors were consumed
    char* dev = static_cast<char*>(L.scratch);
    char* hst = static_cast<char*>(L.pinned);
    auto D = [&](size_t off) { return dev + off; };

    // host inputs: copied straight from the caller's buffers when they are page-locked,
    // else staged through the lane's pinned buffer (one copy together with the descriptors)
    struct HostIn {
        const void* src;
        size_t off, bytes;
        bool detect; // a detection job's samples
    };
    std::vector<HostIn> ins;
    bool direct = false;
    bool stage_split = false; // pageable detection samples staged and uploaded per segment while the batch trains
    if (host) {
        if (!zc_train)
            for (const auto& t : tp) {
                const apsm_job& j = jobs[t.job];
                ins.push_back({j.rx, t.off_rx, sizeof(float2) * size_t(t.det->N) * t.P, false});
                ins.push_back({j.tx, t.off_tx, sizeof(float2) * t.P, false});
            }
        for (const auto& q : dp)
            ins.push_back({jobs[q.job].rx, q.off_rx, sizeof(float2) * size_t(q.det->N) * q.S, true});
        // small batches travel in the one descriptor upload even from page-locked buffers: a
        // host memcpy of a few KB costs less than a copy command per input
        size_t in_bytes = 0;
        for (const auto& in : ins) in_bytes += in.bytes;
        direct = !ins.empty() && in_bytes >= (size_t(256) << 10);
        if (direct)
            for (const auto& in : ins)
                if (in.detect && !is_pinned(in.src)) {
                    direct = false;
                    break;
                }
        // a batch that trains and detects from ordinary (pageable) buffers: the training inputs are
        // staged and uploaded first; the detection samples are staged segment by segment after
        // the training launches and uploaded on the copy stream while the batch trains
        if (!direct && nT > 0 && nD > 0) {
            size_t det_bytes = 0;
            for (const auto& in : ins) det_bytes += in.detect ? in.bytes : 0;
            stage_split = det_bytes >= kZeroCopyMin;
        }
        // staged: every input (no direct copies), or the training inputs of a direct or split batch
        // -- many small copies cost more per byte than helper threads' memcpy plus one upload
        std::vector<Stager::Range> pieces;
        pieces.reserve(ins.size());
        for (const auto& in : ins)
            if (!(direct || stage_split) || !in.detect)
                pieces.push_back({hst + in.off, static_cast<const char*>(in.src), in.bytes});
        stager.begin(pieces); // joined before the upload; the descriptors are written meanwhile
    }

    // ---------- descriptors ----------
    auto* h_tj = reinterpret_cast<BatchTrainJob*>(hst + off_tj);
    auto* h_dj = reinterpret_cast<BatchDetectJob*>(hst + off_dj);
    auto* h_pj = reinterpret_cast<BatchPackJob*>(hst + off_pj);
    auto* h_ci = reinterpret_cast<BatchCopyJob*>(hst + off_ci);
    auto* h_co = reinterpret_cast<BatchCopyJob*>(hst + off_co);
    size_t ipack = 0, icopy = 0;
    int max_len = 0, max_np = 1, max_n = 1, max_pairs_in = 0, max_pairs_out = 0;
    // antenna classes of the kernel-column launches; the training samples are packed in class
    // order, so that each class's pack is one contiguous launch
    auto cls_of = [](int n) { return n <= 4 ? 0 : n <= 8 ? 1 : n <= 16 ? 2 : n <= 32 ? 3 : 4; };
    struct PackClass {
        int first = 0, count = 0, max_len = 0, max_n = 1;
    };
    PackClass pcls[5];
    for (size_t k = 0; k < nT; ++k) ++pcls[cls_of(int(tp[k].det->N))].count;
    for (int c = 1; c < 5; ++c) pcls[c].first = pcls[c - 1].first + pcls[c - 1].count;
    int pfill[5];
    for (int c = 0; c < 5; ++c) pfill[c] = pcls[c].first;
    for (size_t k = 0; k < nT; ++k) {
        TrainPlan& t = tp[k];
        PoolDet& d = *t.det;
        const apsm_job& j = jobs[t.job];
        if (!arena) std::memcpy(hst + t.off_steps, t.steps->data(), sizeof(TrainStep) * t.steps->size());
        const float2* rx = !host ? reinterpret_cast<const float2*>(j.rx)
                                 : zc_train ? static_cast<const float2*>(t.zc_rx) : reinterpret_cast<const float2*>(D(t.off_rx));
        const float2* tx = !host ? reinterpret_cast<const float2*>(j.tx)
                                 : zc_train ? static_cast<const float2*>(t.zc_tx) : reinterpret_cast<const float2*>(D(t.off_tx));
        auto* Y = reinterpret_cast<float2*>(D(t.off_Y));
        auto* nrm = reinterpret_cast<float*>(D(t.off_nrm));
        auto* yv = reinterpret_cast<float*>(D(t.off_y));
        auto* av = reinterpret_cast<float*>(D(t.off_a));
        if (t.usedP > 0) {
            h_ci[icopy++] = BatchCopyJob{d.Y, d.nrm, d.y, d.a, Y, nrm, yv, av, int(t.usedP), int(d.Np)};
            max_pairs_in = std::max(max_pairs_in, int(t.usedP));
        }
        const int* perm = cfg.shuffle ? reinterpret_cast<const int*>(D(t.perm_off)) : nullptr;
        {
            PackClass& pc = pcls[cls_of(int(d.N))];
            h_pj[pfill[cls_of(int(d.N))]++] =
                BatchPackJob{rx, tx, perm, Y + size_t(t.usedP) * d.Np, nrm + t.usedP, yv + 2 * t.usedP,
                             av + 2 * t.usedP, int(t.P), int(d.N), int(d.Np)};
            pc.max_len = std::max(pc.max_len, int(t.P));
            pc.max_n = std::max(pc.max_n, int(d.N));
            ++ipack;
        }
        max_len = std::max(max_len, int(t.P));
        max_np = std::max(max_np, int(d.Np));
        max_n = std::max(max_n, int(d.N));
        BatchTrainJob tj{};
        tj.Y = Y;
        tj.nrm = nrm;
        tj.y = yv;
        tj.a = av;
        tj.w = d.w;
        tj.r = d.r;
        tj.Kc = reinterpret_cast<const float4*>(D(t.off_kc));
        tj.steps = arena ? sched_arena.p + *t.steps_dev : reinterpret_cast<const TrainStep*>(D(t.off_steps));
        tj.n_steps = int(t.steps->size());
        tj.nP = int(t.nP);
        tj.N = int(d.N);
        tj.Np = int(d.Np);
        tj.capP = int(d.capP);
        tj.n_first = int(t.n_first);
        tj.used_beforeP = int(t.usedP);
        tj.kc_base = t.kc_base;
        tj.ew = d.ew;
        tj.fresh = t.fresh ? 1 : 0;
        tj.pro = t.pro_n > 0 ? reinterpret_cast<float2*>(D(t.off_pro)) : nullptr;
        tj.pro_w = t.pro_w;
        tj.pro_lo = t.pro_lo;
        tj.pro_hi = int(t.usedP);
        tj.pro_stride = t.pro_stride;
        h_tj[k] = tj;
        h_co[k] = BatchCopyJob{Y + size_t(t.lo_new) * d.Np, nrm + t.lo_new, yv + 2 * t.lo_new, av + 2 * t.lo_new,
                               d.Y, d.nrm, d.y, d.a, int(t.usedP_new), int(d.Np)};
        max_pairs_out = std::max(max_pairs_out, int(t.usedP_new));
    }
    for (auto& kv : perm_off) std::memcpy(hst + kv.second, perms[kv.first].data(), sizeof(int) * kv.first);
    const size_t pack_train = ipack;
    // kernel-column launches, one per antenna class and form: the CUDA-core kernel (rows of the
    // class's size in registers) and the tensor-core kernel (operands of the class's Kp)
    struct KcolClass {
        int first = 0, count = 0, max_cols = 0, max_n = 1;
        int tc_first = 0, tc_count = 0, tc_units = 0, tc_chunks = 0, tc_kp = 0, tc_prefix = 0;
    };
    KcolClass kcls[5];
    {
        for (size_t k = 0; k < nT; ++k) {
            KcolClass& kc = kcls[cls_of(int(tp[k].det->N))];
            ++(tp[k].kc_tc ? kc.tc_count : kc.count);
        }
        for (int c = 1; c < 5; ++c) {
            kcls[c].first = kcls[c - 1].first + kcls[c - 1].count;
            kcls[c].tc_first = kcls[c - 1].tc_first + kcls[c - 1].tc_count;
            kcls[c].tc_prefix = kcls[c - 1].tc_prefix + kcls[c - 1].tc_count + 1;
        }
        int fill[5], tc_fill[5];
        for (int c = 0; c < 5; ++c) {
            fill[c] = kcls[c].first;
            tc_fill[c] = kcls[c].tc_first;
        }
        auto* h_ko = reinterpret_cast<int*>(hst + off_ko);
        auto* h_kt = reinterpret_cast<BatchKcolTcJob*>(hst + off_kt);
        auto* h_ktp = reinterpret_cast<int*>(hst + off_ktp);
        for (size_t k = 0; k < nT; ++k) {
            const int c = cls_of(int(tp[k].det->N));
            KcolClass& kc = kcls[c];
            const TrainPlan& t = tp[k];
            if (!t.kc_tc) {
                h_ko[fill[c]++] = int(k);
                kc.max_cols = std::max(kc.max_cols, int(t.nP - t.n_first));
                kc.max_n = std::max(kc.max_n, int(t.det->N));
                continue;
            }
            const int i = tc_fill[c]++;
            BatchKcolTcJob kj{};
            kj.Y = reinterpret_cast<const float2*>(D(t.off_Y));
            kj.nrm = reinterpret_cast<const float*>(D(t.off_nrm));
            kj.Kc = reinterpret_cast<float4*>(D(t.off_kc));
            kj.a_ops = reinterpret_cast<uint8_t*>(D(t.off_kca));
            kj.b_ops = reinterpret_cast<uint8_t*>(D(t.off_kcb));
            kj.a_nrm = reinterpret_cast<float*>(D(t.off_kcn));
            kj.nP = int(t.nP);
            kj.N = int(t.det->N);
            kj.Np = int(t.det->Np);
            kj.Kp = t.kc_Kp;
            kj.capP = int(t.det->capP);
            kj.n_first = int(t.n_first);
            kj.a_tiles = t.kc_a_tiles;
            kj.b_chunks = t.kc_b_chunks;
            kj.kc_base = t.kc_base;
            kj.ewl2 = t.det->ew * 1.4426950408889634f;
            h_kt[i] = kj;
            // chunk prefix of the class: one entry per job plus the total
            h_ktp[kc.tc_prefix + (i - kc.tc_first)] = kc.tc_chunks;
            kc.tc_chunks += t.kc_b_chunks;
            kc.tc_units = std::max(kc.tc_units, t.kc_a_tiles + t.kc_b_chunks);
            kc.tc_kp = std::max(kc.tc_kp, t.kc_Kp);
        }
        for (int c = 0; c < 5; ++c)
            if (kcls[c].tc_count > 0) h_ktp[kcls[c].tc_prefix + kcls[c].tc_count] = kcls[c].tc_chunks;
    }
    for (size_t k = 0; k < nD; ++k) {
        DetectPlan& q = dp[k];
        PoolDet& d = *q.det;
        const apsm_job& j = jobs[q.job];
        const float2* rx = host ? reinterpret_cast<const float2*>(D(q.off_rx)) : reinterpret_cast<const float2*>(j.rx);
        auto* ns = q.gram ? reinterpret_cast<float*>(D(q.off_nrm)) : nullptr;
        float2* out = !host ? reinterpret_cast<float2*>(j.est)
                            : zc_est ? static_cast<float2*>(q.zc_est) : reinterpret_cast<float2*>(D(q.off_est));
        const bool split = det_parts > 1 && !q.gram;
        h_dj[k] = BatchDetectJob{rx,       d.Y,       d.nrm, d.a,  d.w, out, int(q.S), int(q.Mp), int(d.N), int(d.Np),
                                 d.ew,     split ? reinterpret_cast<float2*>(D(q.off_part)) : nullptr,
                                 split ? reinterpret_cast<int*>(D(q.off_cnt)) : nullptr};
        if (q.gram) {
            BatchGramJob g{};
            g.rx = rx;
            g.nrm_s = ns;
            g.w = d.w;
            g.lin = reinterpret_cast<float2*>(D(q.off_lin));
            g.a_ops = reinterpret_cast<uint8_t*>(D(q.off_aops));
            g.Yd = d.Y;
            g.nrm_d = d.nrm;
            g.a = d.a;
            g.b_ops = reinterpret_cast<uint8_t*>(D(q.off_bops));
            g.bx = reinterpret_cast<float*>(D(q.off_bx));
            g.out = out;
            g.S = int(q.S);
            g.N = int(d.N);
            g.Np = int(d.Np);
            g.Kp = q.Kp;
            g.Mp = int(q.Mp);
            g.n_chunks = q.chunks;
            g.ew2 = d.ew * 1.4426950408889634f;
            reinterpret_cast<BatchGramJob*>(hst + off_gj)[k - (nD - nG)] = g;
        }
    }
    // tile prefixes of the tensor-core classes (one segment per class)
    std::vector<std::array<int, 6>> gseg; // k0, k1, prefix offset, total tiles, max tiles, max chunks
    {
        int* pre = reinterpret_cast<int*>(hst + off_gp);
        size_t k = nD - nG, po = 0;
        while (k < nD) {
            size_t k1 = k;
            int acc = 0, mt = 0, mc = 0;
            while (k1 < nD && dp[k1].cls == dp[k].cls) {
                pre[po + (k1 - k)] = acc;
                acc += dp[k1].tiles;
                mt = std::max(mt, dp[k1].tiles);
                mc = std::max(mc, dp[k1].chunks);
                ++k1;
            }
            pre[po + (k1 - k)] = acc;
            gseg.push_back({int(k), int(k1), int(po), acc, mt, mc});
            po += k1 - k + 1;
            k = k1;
        }
    }

    const double t_desc = trace ? host_us() : 0.0;
    // ---------- enqueue ----------
    cudaStream_t s = L.stream;
    std::memset(hst + off_counter, 0, off_dcnt - off_counter + dcnt_bytes);
    stager.wait();
    const double t_stage = trace ? host_us() : 0.0;
    if (trace) POOL_CK(cudaEventRecord(L.tr[0], s));
    // a batch that trains and detects from page-locked buffers (or stages pageable ones per
    // segment) copies the detection samples on the lane's copy stream while it trains: after
    // the upload of the descriptors and training inputs (which would otherwise share the link
    // with them and delay the training) and after the lane's earlier work (the scratch is
    // free); the detections wait for them
    const bool overlap = (direct || stage_split) && nT > 0 && nD > 0;
    POOL_CK(cudaMemcpyAsync(dev, hst, (direct || stage_split) ? off_det_in : desc_bytes, cudaMemcpyHostToDevice, s));
    if (direct && !overlap)
        for (const auto& in : ins)
            if (in.detect) POOL_CK(cudaMemcpyAsync(dev + in.off, in.src, in.bytes, cudaMemcpyHostToDevice, s));
    // (the copy commands themselves are issued after the training launches: a host call per
    // input would otherwise hold the training back)
    if (overlap) POOL_CK(cudaEventRecord(L.ev_start, s));
    POOL_CK(cudaEventRecord(L.desc_copied, s));
    L.have_train = timing && nT > 0;
    L.have_detect = timing && nD > 0;
    for (PoolDet* d : resets) {
        POOL_CK(cudaMemsetAsync(d->w, 0, sizeof(float) * 2 * d->N, s));
        POOL_CK(cudaMemsetAsync(d->r, 0, sizeof(float) * 2 * d->N, s));
        d->used = 0;
    }
    int* d_counter = reinterpret_cast<int*>(D(off_counter));
    int* d_err = d_counter + 4;

    L.err = d_err;
    L.launches = 0;
    if (trace) POOL_CK(cudaEventRecord(L.tr[1], s));
    if (nT > 0) {
        if (timing) POOL_CK(cudaEventRecord(L.ev[0], s));
        POOL_CK(launch_batch_copy(reinterpret_cast<const BatchCopyJob*>(D(off_ci)), int(nCopyIn), max_pairs_in, max_np, s));
        L.launches += nCopyIn > 0 && max_pairs_in > 0;
    }
    // training samples (detection reads its samples as the caller holds them).  With host inputs
    // on the copy stream (overlap), each class is packed there -- from page-locked buffers the
    // pack reads over the link -- while the previous class's kernel columns run, and the detection
    // samples follow the packs on that stream, so they do not share the link with them
    const auto* d_pj = reinterpret_cast<const BatchPackJob*>(D(off_pj));
    bool packed_on_copy[5] = {};
    if (pack_train > 0 && overlap) {
        POOL_CK(cudaStreamWaitEvent(L.copy_stream, L.ev_start, 0));
        for (int c = 0; c < 5; ++c) {
            if (pcls[c].count == 0 || pcls[c].max_len <= 0) continue;
            // (inputs read over the link: two blocks per SM -- few blocks in flight saturate the
            // link, and the kernel columns of the classes packed before run beside them)
            POOL_CK(launch_batch_pack(d_pj + pcls[c].first, pcls[c].count, pcls[c].max_len, pcls[c].max_n,
                                      L.copy_stream, zc_train ? 2 * sms : 0));
            POOL_CK(cudaEventRecord(L.ev_pack[c], L.copy_stream));
            packed_on_copy[c] = true;
            ++L.launches;
        }
        if (trace) POOL_CK(cudaEventRecord(L.tr_copy[0], L.copy_stream));
    } else if (pack_train > 0) {
        POOL_CK(launch_batch_pack(d_pj, int(pack_train), max_len, max_n, s));
        L.launches += max_len > 0;
    }
    if (trace) POOL_CK(cudaEventRecord(L.tr[2], s));
    if (nT > 0) {
        const auto* d_tj = reinterpret_cast<const BatchTrainJob*>(D(off_tj));
        const int* d_ko = reinterpret_cast<const int*>(D(off_ko));
        const auto* d_kt = reinterpret_cast<const BatchKcolTcJob*>(D(off_kt));
        const int* d_ktp = reinterpret_cast<const int*>(D(off_ktp));
        for (int c = 0; c < 5; ++c) {
            const KcolClass& kc = kcls[c];
            if (packed_on_copy[c] && (kc.tc_count > 0 || (kc.count > 0 && kc.max_cols > 0)))
                POOL_CK(cudaStreamWaitEvent(s, L.ev_pack[c], 0));
            if (kc.tc_count > 0) {
                POOL_CK(launch_batch_kcol_tc(d_kt + kc.tc_first, kc.tc_count, kc.tc_units, d_ktp + kc.tc_prefix,
                                             kc.tc_chunks, kc.tc_kp, cm, d_err, s));
                L.launches += 2;
            }
            if (kc.count == 0 || kc.max_cols <= 0) continue;
            // small launches (single train requests): spread each column group's rows over blocks
            int row_split = 1;
            const long long blocks = (long long)kc.count * ((kc.max_cols + batch_kcol_group() - 1) / batch_kcol_group());
            const int passes = int((int(cfg.dict_size) + cm.qP + batch_kcol_rows() - 1) / batch_kcol_rows());
            const long long target = 4LL * std::max(1, sms);
            if (blocks < target)
                row_split = int(std::min<long long>(std::max(passes, 1), (target + blocks - 1) / blocks));
            POOL_CK(launch_batch_kcol(d_tj, d_ko + kc.first, kc.count, kc.max_cols, kc.max_n, row_split, cm, s));
            ++L.launches;
        }
        if (trace) POOL_CK(cudaEventRecord(L.tr[3], s));
        for (int c = 0; c < 5; ++c) // (a class without kernel columns to compute)
            if (packed_on_copy[c]) POOL_CK(cudaStreamWaitEvent(s, L.ev_pack[c], 0));
        const int per_sm = shape.sweep_per_sm > 0 ? std::min(shape.sweep_per_sm, sweep_ctas) : sweep_ctas;
        const int grid = int(std::min<size_t>(nT, size_t(per_sm) * sms));
        if (timing) POOL_CK(cudaEventRecord(L.ev[4], s));
        POOL_CK(launch_batch_sweep(d_tj, int(nT), cm, grid, d_counter, d_err, s));
        if (timing) POOL_CK(cudaEventRecord(L.ev[5], s));
        if (trace) POOL_CK(cudaEventRecord(L.tr[4], s));
        POOL_CK(launch_batch_copy(reinterpret_cast<const BatchCopyJob*>(D(off_co)), int(nT), max_pairs_out, max_np, s));
        L.launches += 1 + (max_pairs_out > 0);
        if (timing) POOL_CK(cudaEventRecord(L.ev[1], s));
        for (const auto& t : tp) t.det->used = 2 * t.usedP_new;
    } else if (trace) {
        POOL_CK(cudaEventRecord(L.tr[3], s));
        POOL_CK(cudaEventRecord(L.tr[4], s));
    }
    if (trace) POOL_CK(cudaEventRecord(L.tr[5], s));
    if (nD > 0) {
        // detection in segments of one launch shape (the CUDA-core classes, then the tensor-core
        // classes); when the samples travel on the copy stream each segment waits for its own
        // only, and each segment's estimates are copied back behind it
        struct Seg {
            size_t k0, k1;
            int g; // index into gseg; -1 for a CUDA-core class
        };
        std::vector<Seg> segs;
        const size_t nC = nD - nG; // CUDA-core jobs come first
        for (size_t k0 = 0; k0 < nC;) {
            size_t k1 = k0;
            while (k1 < nC && dp[k1].cls == dp[k0].cls) ++k1;
            segs.push_back({k0, k1, -1});
            k0 = k1;
        }
        for (size_t g = 0; g < gseg.size(); ++g) segs.push_back({size_t(gseg[g][0]), size_t(gseg[g][1]), int(g)});
        if (overlap && segs.size() > 1) {
            // Order of the segments when their samples come on the copy stream (which also carries
            // the training samples first): each detection waits for its own copies, so this is a
            // two-stage flow shop (copy, then detect) and Johnson's rule orders it -- segments whose
            // copy is shorter than their detection first, by increasing copy time, then the others
            // by decreasing detection time.  Times are estimates: bytes at ~45 GB/s; pair
            // evaluations at ~8e11/s on the tensor cores (the 64-wide operand class at 1.6x the
            // cost) and a fifth of that for the CUDA-core forms.  The estimates do not depend on
            // the order (segments are independent).
            std::vector<std::pair<double, double>> cost(segs.size()); // (copy, detect), seconds
            for (size_t i = 0; i < segs.size(); ++i) {
                double bytes = 0.0, pairs = 0.0;
                for (size_t k = segs[i].k0; k < segs[i].k1; ++k) {
                    bytes += double(sizeof(float2)) * dp[k].det->N * dp[k].S;
                    pairs += double(dp[k].S) * double(dp[k].Mp);
                }
                const double w = segs[i].g < 0 ? 5.0 : (dp[segs[i].k0].Kp > 32 ? 1.6 : 1.0);
                cost[i] = {bytes / 45e9, w * pairs / 8e11};
            }
            std::vector<size_t> ord(segs.size());
            for (size_t i = 0; i < ord.size(); ++i) ord[i] = i;
            std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) {
                const bool fx = cost[x].first < cost[x].second, fy = cost[y].first < cost[y].second;
                if (fx != fy) return fx;
                return fx ? cost[x].first < cost[y].first : cost[x].second > cost[y].second;
            });
            std::vector<Seg> sorted;
            sorted.reserve(segs.size());
            for (size_t i : ord) sorted.push_back(segs[i]);
            segs.swap(sorted);
        }
        if (overlap) {
            while (L.seg_ev.size() < segs.size()) {
                cudaEvent_t e = nullptr;
                POOL_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
                L.seg_ev.push_back(e);
            }
            POOL_CK(cudaStreamWaitEvent(L.copy_stream, L.ev_start, 0));
        }
        // segment i's samples onto the copy stream, then its event; issued just before the
        // segment's detection launches (a detection does not wait for the staging of later segments)
        auto copy_segment = [&](size_t i) -> apsm_status {
            if (stage_split) {
                // the segment's samples (contiguous in the staging layout) in groups of jobs of
                // ~kSplitGroup bytes: a group is staged by the helper threads, then uploaded in
                // one copy while the next group is staged
                std::vector<Stager::Range> pieces;
                size_t lo = dp[segs[i].k0].off_rx, hi = lo;
                for (size_t k = segs[i].k0; k < segs[i].k1; ++k) {
                    const DetectPlan& q = dp[k];
                    const size_t bytes = sizeof(float2) * size_t(q.det->N) * q.S;
                    pieces.push_back({hst + q.off_rx, reinterpret_cast<const char*>(jobs[q.job].rx), bytes});
                    hi = q.off_rx + bytes;
                    if (hi - lo >= kSplitGroup || k + 1 == segs[i].k1) {
                        stager.copy(pieces);
                        POOL_CK(cudaMemcpyAsync(dev + lo, hst + lo, hi - lo, cudaMemcpyHostToDevice, L.copy_stream));
                        pieces.clear();
                        if (k + 1 < segs[i].k1) lo = dp[k + 1].off_rx;
                    }
                }
            } else {
                for (size_t k = segs[i].k0; k < segs[i].k1; ++k) {
                    const DetectPlan& q = dp[k];
                    POOL_CK(cudaMemcpyAsync(dev + q.off_rx, jobs[q.job].rx, sizeof(float2) * size_t(q.det->N) * q.S,
                                            cudaMemcpyHostToDevice, L.copy_stream));
                }
            }
            POOL_CK(cudaEventRecord(L.seg_ev[i], L.copy_stream));
            return APSM_OK;
        };
        // page-locked outputs of a few jobs: one copy each; of many jobs: one copy per segment,
        // scattered by finish() (per-copy cost exceeds a host memcpy then)
        const bool est_out = host && est_bytes > 0;
        bool out_direct = est_out && dp.size() <= kDirectOutJobs;
        for (const auto& q : dp)
            if (out_direct && !is_pinned(jobs[q.job].est)) {
                out_direct = false;
                break;
            }
        if (timing) POOL_CK(cudaEventRecord(L.ev[2], s));
        const auto* d_dj = reinterpret_cast<const BatchDetectJob*>(D(off_dj));
        const auto* d_gj = reinterpret_cast<const BatchGramJob*>(D(off_gj));
        const int* d_gp = reinterpret_cast<const int*>(D(off_gp));
        for (size_t i = 0; i < segs.size(); ++i) {
            const Seg& sg = segs[i];
            if (overlap) {
                const apsm_status st = copy_segment(i);
                if (st != APSM_OK) return st;
                POOL_CK(cudaStreamWaitEvent(s, L.seg_ev[i], 0));
            }
            if (sg.g < 0) {
                int tiles = 0;
                for (size_t k = sg.k0; k < sg.k1; ++k)
                    tiles = std::max(tiles, int((dp[k].S + batch_detect_tile() - 1) / batch_detect_tile()));
                POOL_CK(launch_batch_detect(d_dj + sg.k0, int(sg.k1 - sg.k0), tiles, det_parts, dp[sg.k0].cls, cfg.wL,
                                            cfg.wG, s));
                L.launches += tiles > 0;
            } else {
                // (the operand packing reads the class's samples as the caller holds them)
                const auto& g = gseg[size_t(sg.g)];
                POOL_CK(launch_batch_gram(gram_mode, d_gj + (sg.k0 - nC), g[1] - g[0], g[4], g[5], d_gp + g[2], g[3],
                                          dp[sg.k0].cls, cfg.wL, cfg.wG, d_err, shape.gram_stages, s));
                L.launches += (g[4] > 0) + (g[5] > 0) + (g[3] > 0);
            }
            if (out_direct) {
                for (size_t k = sg.k0; k < sg.k1; ++k)
                    POOL_CK(cudaMemcpyAsync(jobs[dp[k].job].est, D(dp[k].off_est), sizeof(float2) * dp[k].S,
                                            cudaMemcpyDeviceToHost, s));
            } else if (est_out) {
                const size_t lo = dp[sg.k0].off_est, hi = dp[sg.k1 - 1].off_est + sizeof(float2) * dp[sg.k1 - 1].S;
                POOL_CK(cudaMemcpyAsync(static_cast<char*>(L.pinned_out) + (lo - est_begin), D(lo), hi - lo,
                                        cudaMemcpyDeviceToHost, s));
            }
        }
        if (overlap) {
            // (the staging buffer is consumed once the last upload is done)
            if (stage_split) POOL_CK(cudaEventRecord(L.desc_copied, L.copy_stream));
            if (trace) POOL_CK(cudaEventRecord(L.tr_copy[1], L.copy_stream));
        }
        if (est_out && !out_direct)
            for (const auto& q : dp) L.pending.push_back({jobs[q.job].est, q.off_est - est_begin, sizeof(float2) * q.S});
        if (timing) POOL_CK(cudaEventRecord(L.ev[3], s));
    }
    // the error flag of kernels with bounded waits (tensor-core detection) travels back with the
    // batch: finish() reads it without a synchronous copy
    bool any_kc_tc = false;
    for (const auto& t : tp) any_kc_tc = any_kc_tc || t.kc_tc;
    L.err_copied = nG > 0 || any_kc_tc; // only the tensor-core kernels wait on barriers (bounded, flagging expiry)
    if (L.err_copied) POOL_CK(cudaMemcpyAsync(L.err_host, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (trace) {
        POOL_CK(cudaEventRecord(L.tr[6], s));
        L.traced = true;
        L.tr_overlap = overlap && pack_train > 0;
        L.tr_nT = int(nT);
        L.tr_nD = int(nD);
        L.t_run0 = t_run0;
        L.t_run1 = host_us();
        L.t_mark[0] = t_plan - t_run0;
        L.t_mark[1] = t_desc - t_run0;
        L.t_mark[2] = t_stage - t_run0;
    }
    POOL_CK(cudaEventRecord(L.done, s));
    if (mode == APSM_RUN_HOST) return finish(lane_id);
    L.unfinished = mode == APSM_RUN_HOST_ASYNC;
    return APSM_OK;
}

apsm_status apsm_pool::exact_handle(uint32_t N, apsm_detector** out)
{
    auto it = exact_by_n.find(N);
    if (it == exact_by_n.end()) {
        auto* h = new apsm_detector();
        const apsm_status st = h->init(cfg, N, 1);
        if (st != APSM_OK) {
            const std::string msg = h->last_error;
            delete h;
            return fail(st, "normConstraint training detector: " + msg);
        }
        it = exact_by_n.emplace(N, h).first;
    }
    *out = it->second;
    return APSM_OK;
}

// Training jobs of a normConstraint pool, in the batch's order, each on the lane's stream with the
// exact sweep of a single detector of its antenna count: the pool detector's state is converted to
// Dedup rows, trained, and converted back (same dictionary semantics: rows oldest first, a full
// dictionary evicts its oldest rows, a second call continues the window).  The detection jobs are
// returned in `rest`.
apsm_status apsm_pool::train_exact(uint32_t lane_id, const apsm_job* jobs, uint32_t n, int mode,
                                   std::vector<apsm_job>* rest)
{
    apsm_pool* p = this;
    cudaStream_t s = lanes[lane_id].stream;
    const bool host = mode != APSM_RUN_DEVICE;
    rest->clear();
    for (uint32_t i = 0; i < n; ++i) {
        const apsm_job& j = jobs[i];
        if (j.kind != APSM_JOB_TRAIN) {
            rest->push_back(j);
            continue;
        }
        PoolDet& d = dets[j.detector];
        if (j.flags & APSM_JOB_FRESH) {
            POOL_CK(cudaMemsetAsync(d.w, 0, sizeof(float) * 2 * d.N, s));
            POOL_CK(cudaMemsetAsync(d.r, 0, sizeof(float) * 2 * d.N, s));
            d.used = 0;
        }
        if (j.length == 0) continue;
        apsm_detector* h = nullptr;
        apsm_status st = exact_handle(d.N, &h);
        if (st != APSM_OK) return st;
        const int N = int(d.N), Dp = int(h->Dp), Np = int(d.Np);
        // pool state -> rows of the detector
        h->used = d.used;
        POOL_CK(launch_pool_to_rows(d.Y, Np, d.y, d.a, int(d.used), N, Dp, h->dict_X.p, h->dict_nrm.p, h->dict_y.p,
                                    h->dict_a.p, s));
        POOL_CK(cudaMemcpyAsync(h->w.p, d.w, sizeof(float) * 2 * d.N, cudaMemcpyDeviceToDevice, s));
        const float2* rx = reinterpret_cast<const float2*>(j.rx);
        const float2* tx = reinterpret_cast<const float2*>(j.tx);
        if (host) {
            POOL_CK(h->rx_stage.ensure(size_t(d.N) * j.length));
            POOL_CK(h->tx_stage.ensure(j.length));
            POOL_CK(cudaMemcpyAsync(h->rx_stage.p, rx, sizeof(float2) * size_t(d.N) * j.length,
                                    cudaMemcpyHostToDevice, s));
            POOL_CK(cudaMemcpyAsync(h->tx_stage.p, tx, sizeof(float2) * j.length, cudaMemcpyHostToDevice, s));
            rx = h->rx_stage.p;
            tx = h->tx_stage.p;
        }
        st = h->train(rx, tx, j.length, s, nullptr);
        if (st != APSM_OK) return fail(st, "normConstraint training: " + h->last_error);
        POOL_CK(cudaStreamSynchronize(s));
        st = h->check_train_error();
        if (st != APSM_OK) return fail(st, h->last_error);
        // rows -> pool state (the residual weights of the incremental sweep are not used by
        // normConstraint pools)
        POOL_CK(launch_rows_to_pool(h->dict_X.p, h->dict_nrm.p, h->dict_y.p, h->dict_a.p, int(h->used), N, Dp, Np,
                                    d.Y, d.nrm, d.y, d.a, s));
        POOL_CK(cudaMemcpyAsync(d.w, h->w.p, sizeof(float) * 2 * d.N, cudaMemcpyDeviceToDevice, s));
        d.used = h->used;
    }
    return APSM_OK;
}

// Launch-shape autotuner: the batch is run once per candidate of each knob
// that it exercises (one knob at a time, the others at their current values),
// the GPU time from its first to its last kernel compared, and the fastest
// candidate kept.  The detectors the batch trains get their resident state back
// after every trial and at the end, so the call leaves every detector as it
// found it; no knob changes any result (each is a launch shape over the same
// per-job arithmetic).
apsm_status apsm_pool::autotune(uint32_t lane_id, const apsm_job* jobs, uint32_t n, int mode, std::string* report)
{
    apsm_pool* p = this;
    Lane& L = lanes[lane_id];
    if (!L.pending.empty() || L.unfinished) {
        apsm_status st = finish(lane_id);
        if (st != APSM_OK) return st;
    }
    bool any_train = false, any_gram = false, any_core = false;
    std::vector<uint32_t> ids;
    for (uint32_t i = 0; i < n; ++i) {
        const apsm_job& j = jobs[i];
        if (j.detector >= dets.size() || !dets[j.detector].live)
            return fail(APSM_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": unknown detector");
        if (j.kind == APSM_JOB_TRAIN) {
            if (std::find(ids.begin(), ids.end(), j.detector) == ids.end()) ids.push_back(j.detector);
            any_train = any_train || j.length > 0;
        } else if (j.kind == APSM_JOB_DETECT && j.length > 0) {
            const bool gram = cfg.detect_mode != DetectMode::Exact && dets[j.detector].N <= 32;
            any_gram = any_gram || gram;
            any_core = any_core || !gram;
        }
    }
    // every lane idle: their batches may read the detectors being saved
    for (auto& l : lanes) POOL_CK(cudaStreamSynchronize(l.stream));
    size_t total = 0;
    for (uint32_t id : ids) total += dets[id].bytes;
    char* save = nullptr;
    if (total > 0) POOL_CK(cudaMalloc(&save, total));
    std::vector<uint32_t> used0;
    {
        size_t o = 0;
        for (uint32_t id : ids) {
            cudaError_t e = cudaMemcpy(save + o, dets[id].mem, dets[id].bytes, cudaMemcpyDeviceToDevice);
            if (e != cudaSuccess) {
                cudaFree(save);
                return cuda_fail(e, "cudaMemcpy (autotune save)");
            }
            used0.push_back(dets[id].used);
            o += dets[id].bytes;
        }
    }
    auto restore = [&]() -> cudaError_t {
        size_t o = 0;
        for (size_t k = 0; k < ids.size(); ++k) {
            PoolDet& d = dets[ids[k]];
            cudaError_t e = cudaMemcpy(d.mem, save + o, d.bytes, cudaMemcpyDeviceToDevice);
            if (e != cudaSuccess) return e;
            d.used = used0[k];
            o += d.bytes;
        }
        return cudaSuccess;
    };
    const bool timing0 = timing;
    timing = true;
    // GPU time of one run of the batch (best of two), first kernel to last
    auto trial = [&](float* ms) -> apsm_status {
        *ms = 0.f;
        float best = -1.f;
        for (int rep = 0; rep < 2; ++rep) {
            cudaError_t e = restore();
            if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy (autotune restore)");
            apsm_status st = run(lane_id, jobs, n, mode);
            if (st == APSM_OK && mode != APSM_RUN_HOST) st = finish(lane_id);
            if (st != APSM_OK) return st;
            float t = 0.f;
            cudaEvent_t a = L.have_train ? L.ev[0] : L.ev[2];
            cudaEvent_t b = L.have_detect ? L.ev[3] : L.ev[1];
            if (!L.have_train && !L.have_detect) return APSM_OK;
            e = cudaEventElapsedTime(&t, a, b);
            if (e != cudaSuccess) return cuda_fail(e, "cudaEventElapsedTime (autotune)");
            if (best < 0.f || t < best) best = t;
        }
        *ms = best;
        return APSM_OK;
    };
    std::string rep = "{\"trials\": [";
    bool first = true;
    apsm_status st = APSM_OK;
    auto tune = [&](const char* name, int* knob, const std::vector<int>& cands) {
        if (st != APSM_OK || cands.size() < 2) return;
        int best_v = *knob;
        float best_ms = -1.f;
        for (int v : cands) {
            *knob = v;
            float ms = 0.f;
            st = trial(&ms);
            if (st != APSM_OK) return;
            rep += std::string(first ? "" : ", ") + "{\"" + name + "\": " + std::to_string(v) + ", \"ms\": " +
                   std::to_string(ms) + "}";
            first = false;
            if (best_ms < 0.f || ms < best_ms) {
                best_ms = ms;
                best_v = v;
            }
        }
        *knob = best_v;
    };
    if (any_train) {
        std::vector<int> c;
        for (int v = 1; v <= sweep_ctas; ++v) c.push_back(v);
        tune("sweep_ctas_per_sm", &shape.sweep_per_sm, c);
    }
    if (any_gram) tune("gram_stages", &shape.gram_stages, {2, 3});
    if (any_core) tune("detect_blocks_per_sm", &shape.detect_blocks_per_sm, {1, 2, 4, 8, 16});
    timing = timing0;
    const cudaError_t e = restore();
    cudaFree(save);
    if (st != APSM_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy (autotune restore)");
    rep += "], \"sweep_ctas_per_sm\": " + std::to_string(shape.sweep_per_sm) +
           ", \"gram_stages\": " + std::to_string(shape.gram_stages) +
           ", \"detect_blocks_per_sm\": " + std::to_string(shape.detect_blocks_per_sm) + "}";
    if (report) *report = rep;
    return APSM_OK;
}

apsm_status apsm_pool::finish(uint32_t lane_id)
{
    apsm_pool* p = this;
    Lane& L = lanes[lane_id];
    const double t0 = trace ? host_us() : 0.0;
    POOL_CK(cudaEventSynchronize(L.done));
    L.unfinished = false;
    const double t1 = trace ? host_us() : 0.0;
    {
        std::vector<Stager::Range> pieces;
        pieces.reserve(L.pending.size());
        for (const auto& c : L.pending)
            pieces.push_back({static_cast<char*>(c.dst), static_cast<const char*>(L.pinned_out) + c.off, c.bytes});
        stager.copy(pieces);
    }
    L.pending.clear();
    const apsm_status st = check_lane(lane_id);
    if (trace && L.traced) {
        // one line per batch: lane, jobs, host run() time, host gap until finish(), finish's wait and rest,
        // GPU: inputs copied, packed, kernel columns, sweep, dictionary copied back, detected (+ results
        // copied) -- microseconds
        // (copy stream, host-input batches: training samples packed and detection samples in, from
        // the batch's first GPU mark; -1 otherwise)
        float g[6] = {0, 0, 0, 0, 0, 0}, gc[2] = {-1e-3f, -1e-3f};
        for (int k = 0; k < 6; ++k)
            if (cudaEventElapsedTime(&g[k], L.tr[k], L.tr[k + 1]) != cudaSuccess) g[k] = -1e-3f;
        for (int k = 0; k < 2 && L.tr_overlap; ++k)
            if (cudaEventElapsedTime(&gc[k], L.tr[0], L.tr_copy[k]) != cudaSuccess) gc[k] = -1e-3f;
        cudaGetLastError();
        std::fprintf(trace, "%u %d %d %.1f %.1f %.1f %.1f %.1f %.1f %.1f %.1f %.1f %.1f %.1f %.1f %.1f %.1f %.1f\n",
                     lane_id, L.tr_nT, L.tr_nD, L.t_run1 - L.t_run0, t0 - L.t_run1, t1 - t0, host_us() - t1,
                     1e3 * g[0], 1e3 * g[1], 1e3 * g[2], 1e3 * g[3], 1e3 * g[4], 1e3 * g[5], L.t_mark[0], L.t_mark[1],
                     L.t_mark[2], 1e3 * gc[0], 1e3 * gc[1]);
        L.traced = false;
    }
    return st;
}

apsm_status apsm_pool::check_lane(uint32_t lane_id)
{
    apsm_pool* p = this;
    Lane& L = lanes[lane_id];
    if (!L.err || !L.err_host || !L.err_copied) return APSM_OK;
    const int h = *static_cast<volatile int*>(L.err_host); // copied by the batch before its done event
    if (h) return fail(APSM_ERR_CUDA, "a bounded wait in a tensor-core kernel expired (results of the batch are invalid)");
    return APSM_OK;
}

// ==================================================================== ABI ==

namespace {
void copy_err(char* err, size_t errlen, const std::string& msg)
{
    if (err && errlen) {
        std::strncpy(err, msg.c_str(), errlen - 1);
        err[errlen - 1] = 0;
    }
}
} // namespace

extern "C" apsm_status apsm_pool_create(const char* algorithm_json, uint64_t hbm_budget_bytes, uint32_t lanes,
                                        apsm_pool** out, char* err, size_t errlen)
{
    if (!algorithm_json || !out) {
        copy_err(err, errlen, "null argument");
        return APSM_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (lanes == 0 || lanes > 64) {
        copy_err(err, errlen, "lanes must be in [1, 64]");
        return APSM_ERR_INVALID_ARGUMENT;
    }
    Config cfg;
    try {
        cfg = parse_config(algorithm_json);
    } catch (const std::exception& e) {
        copy_err(err, errlen, e.what());
        return APSM_ERR_INVALID_CONFIG;
    }
    std::string why;
    if (cfg.otype != "APSM") why = "the detector pool runs APSM detectors only";
    else if (cfg.lls_init) why = "llsInitialization is not available in the detector pool";
    else if (!(cfg.variance > 0.f)) why = "the detector pool needs gaussianKernelVariance > 0";
    else if (cfg.step % 2 != 0 || cfg.step == 0 || cfg.step > 8) why = "the detector pool needs an even sampleStep <= 8";
    else if (cfg.dict_size < cfg.window + cfg.step / 2) why = "the detector pool needs dictionarySize >= windowSize + sampleStep / 2";
    else if (cfg.window == 0) why = "windowSize must be >= 1";
    if (!why.empty()) {
        copy_err(err, errlen, why);
        return APSM_ERR_UNSUPPORTED;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        copy_err(err, errlen, "no CUDA device available");
        return APSM_ERR_NO_DEVICE;
    }
    auto* p = new apsm_pool();
    p->cfg = cfg;
    switch (cfg.detect_mode) {
    case DetectMode::GramBF16: p->gram_mode = kBF16; break;
    case DetectMode::GramBF16x3: p->gram_mode = kBF16x3; break;
    case DetectMode::GramTF32: p->gram_mode = kTF32; break;
    default: p->gram_mode = kTF32x3; break;
    }
    p->budget = hbm_budget_bytes;
    BatchCommon& cm = p->cm;
    cm.wL = cfg.wL;
    cm.wG = cfg.wG;
    cm.eB = cfg.eB;
    cm.qP = int(cfg.window);
    cm.sp = int(cfg.step / 2);
    cm.LB = cm.qP + cm.sp;
    cm.XSP = cm.qP + 3 * cm.sp;
    cm.XSPp = int(round_up(uint32_t(cm.XSP) + 1, 4));
    cm.Np = 32; // sweep shared memory sized for N <= 32; larger N re-sizes at add
    auto failp = [&](const std::string& m, apsm_status st) {
        copy_err(err, errlen, m);
        delete p;
        return st;
    };
    cudaDeviceProp prop;
    if (cudaGetDevice(&p->device) != cudaSuccess || cudaGetDeviceProperties(&prop, p->device) != cudaSuccess)
        return failp("cudaGetDeviceProperties failed", APSM_ERR_CUDA);
    if (prop.major < 10) return failp("an sm_100 (Blackwell) device is required", APSM_ERR_NO_DEVICE);
    p->sms = prop.multiProcessorCount;
    {
        cudaMemPoolProps mp = {};
        mp.allocType = cudaMemAllocationTypePinned;
        mp.handleTypes = cudaMemHandleTypeNone;
        mp.location.type = cudaMemLocationTypeDevice;
        mp.location.id = p->device;
        if (cudaMemPoolCreate(&p->mempool, &mp) != cudaSuccess) return failp("cudaMemPoolCreate failed", APSM_ERR_CUDA);
        uint64_t keep = ~0ull; // released memory stays with the pool for the next growth
        cudaMemPoolSetAttribute(p->mempool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    p->lanes.resize(lanes);
    for (auto& l : p->lanes) {
        if (cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking) != cudaSuccess)
            return failp("cudaStreamCreate failed", APSM_ERR_CUDA);
        for (auto& e : l.ev)
            if (cudaEventCreate(&e) != cudaSuccess) return failp("cudaEventCreate failed", APSM_ERR_CUDA);
        if (cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&l.desc_copied, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&l.ev_start, cudaEventDisableTiming) != cudaSuccess)
            return failp("cudaEventCreate failed", APSM_ERR_CUDA);
        if (cudaStreamCreateWithFlags(&l.copy_stream, cudaStreamNonBlocking) != cudaSuccess)
            return failp("cudaStreamCreate failed", APSM_ERR_CUDA);
        for (auto& e : l.ev_pack)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
                return failp("cudaEventCreate failed", APSM_ERR_CUDA);
        for (auto& e : l.tr)
            if (cudaEventCreate(&e) != cudaSuccess) return failp("cudaEventCreate failed", APSM_ERR_CUDA);
        for (auto& e : l.tr_copy)
            if (cudaEventCreate(&e) != cudaSuccess) return failp("cudaEventCreate failed", APSM_ERR_CUDA);
        if (cudaMallocHost(reinterpret_cast<void**>(&l.err_host), sizeof(int)) != cudaSuccess)
            return failp("cudaMallocHost failed", APSM_ERR_CUDA);
        *l.err_host = 0;
        cudaEventRecord(l.done, l.stream);
        cudaEventRecord(l.desc_copied, l.stream);
    }
    if (const char* f = std::getenv("APSM_POOL_KCOL")) {
        if (std::strcmp(f, "cuda") == 0) p->kcol_tc_off = true;
        if (std::strcmp(f, "tensor") == 0) p->kcol_tc_min_n = 1;
    }
    if (const char* path = std::getenv("APSM_POOL_TRACE")) {
        p->trace = std::fopen(path, "w");
        if (p->trace)
            std::fprintf(p->trace, "# lane n_train n_detect run_us gap_us fin_wait_us fin_rest_us gpu_inputs_us "
                                   "gpu_pack_us gpu_kcol_us gpu_sweep_us gpu_copyout_us gpu_detect_us "
                                   "run_planned_us run_described_us run_staged_us gpu_packed_at_us "
                                   "gpu_detect_inputs_at_us\n");
    }
    if (cudaStreamCreateWithFlags(&p->sched_stream, cudaStreamNonBlocking) != cudaSuccess)
        return failp("cudaStreamCreate failed", APSM_ERR_CUDA);
    if (batch_sweep_occupancy(cm, &p->sweep_ctas) != cudaSuccess || p->sweep_ctas < 1)
        return failp("the training sweep does not fit an SM", APSM_ERR_UNSUPPORTED);
    *out = p;
    return APSM_OK;
}

extern "C" void apsm_pool_destroy(apsm_pool* p) { delete p; }

extern "C" const char* apsm_pool_last_error(const apsm_pool* p) { return p ? p->last_error.c_str() : "null handle"; }

extern "C" apsm_status apsm_pool_add(apsm_pool* p, uint32_t num_antennas, uint32_t* detector)
{
    if (!p || !detector) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(p->mu);
    if (num_antennas == 0) return p->fail(APSM_ERR_INVALID_ARGUMENT, "num_antennas must be >= 1");
    if (num_antennas > uint32_t(kMaxFeatures / 2))
        return p->fail(APSM_ERR_UNSUPPORTED, "num_antennas must be <= " + std::to_string(kMaxFeatures / 2));
    PoolDet d;
    d.N = num_antennas;
    d.Np = round_up(num_antennas, 2);
    d.capP = p->cfg.dict_size;
    d.cap = 2 * d.capP;
    d.ew = -0.5f / (p->cfg.variance * float(num_antennas * num_antennas));
    size_t off[6];
    d.bytes = resident_layout(d.N, d.capP, off);
    if (p->budget && p->in_use() + d.bytes > p->budget)
        return p->fail(APSM_ERR_OUT_OF_MEMORY, "detector state of " + std::to_string(d.bytes) +
                                                   " bytes exceeds the pool's HBM budget");
    if (int(d.Np) > p->cm.Np) {
        BatchCommon cm2 = p->cm;
        cm2.Np = int(d.Np);
        int ctas = 0;
        if (batch_sweep_occupancy(cm2, &ctas) != cudaSuccess || ctas < 1)
            return p->fail(APSM_ERR_UNSUPPORTED, "the training sweep does not fit an SM for this antenna count");
        for (auto& l : p->lanes) cudaStreamSynchronize(l.stream);
        p->cm = cm2;
        p->sweep_ctas = ctas;
    }
    cudaError_t e = cudaMalloc(&d.mem, d.bytes);
    if (e != cudaSuccess) return p->cuda_fail(e, "cudaMalloc(detector state)");
    char* m = static_cast<char*>(d.mem);
    d.Y = reinterpret_cast<float2*>(m + off[0]);
    d.nrm = reinterpret_cast<float*>(m + off[1]);
    d.y = reinterpret_cast<float*>(m + off[2]);
    d.a = reinterpret_cast<float*>(m + off[3]);
    d.w = reinterpret_cast<float*>(m + off[4]);
    d.r = reinterpret_cast<float*>(m + off[5]);
    e = cudaMemset(d.mem, 0, d.bytes);
    if (e != cudaSuccess) {
        cudaFree(d.mem);
        return p->cuda_fail(e, "cudaMemset(detector state)");
    }
    d.live = true;
    p->resident += d.bytes;
    for (size_t i = 0; i < p->dets.size(); ++i)
        if (!p->dets[i].live && !p->dets[i].mem) {
            p->dets[i] = d;
            *detector = uint32_t(i);
            return APSM_OK;
        }
    p->dets.push_back(d);
    *detector = uint32_t(p->dets.size() - 1);
    return APSM_OK;
}

extern "C" apsm_status apsm_pool_remove(apsm_pool* p, uint32_t detector)
{
    if (!p) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(p->mu);
    if (detector >= p->dets.size() || !p->dets[detector].live)
        return p->fail(APSM_ERR_INVALID_ARGUMENT, "unknown detector");
    for (auto& l : p->lanes) cudaStreamSynchronize(l.stream);
    PoolDet& d = p->dets[detector];
    cudaFree(d.mem);
    p->resident -= d.bytes;
    d = PoolDet();
    return APSM_OK;
}

extern "C" apsm_status apsm_pool_reset(apsm_pool* p, uint32_t detector)
{
    if (!p) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(p->mu);
    if (detector >= p->dets.size() || !p->dets[detector].live)
        return p->fail(APSM_ERR_INVALID_ARGUMENT, "unknown detector");
    PoolDet& d = p->dets[detector];
    for (auto& l : p->lanes) cudaStreamSynchronize(l.stream);
    cudaError_t e = cudaMemset(d.mem, 0, d.bytes);
    if (e != cudaSuccess) return p->cuda_fail(e, "cudaMemset(detector state)");
    d.used = 0;
    return APSM_OK;
}

extern "C" apsm_status apsm_pool_run(apsm_pool* p, uint32_t lane, const apsm_job* jobs, uint32_t n_jobs,
                                     int device_buffers)
{
    if (!p) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(p->mu);
    if (lane >= p->lanes.size()) return p->fail(APSM_ERR_INVALID_ARGUMENT, "lane out of range");
    if (n_jobs > 0 && !jobs) return p->fail(APSM_ERR_INVALID_ARGUMENT, "null job list");
    if (device_buffers < 0 || device_buffers > 2) return p->fail(APSM_ERR_INVALID_ARGUMENT, "unknown run mode");
    return p->run(lane, jobs, n_jobs, device_buffers);
}

extern "C" apsm_status apsm_pool_reserve(apsm_pool* p, uint32_t lane, const apsm_job* jobs, uint32_t n_jobs,
                                         int mode)
{
    if (!p) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(p->mu);
    if (lane >= p->lanes.size()) return p->fail(APSM_ERR_INVALID_ARGUMENT, "lane out of range");
    if (n_jobs > 0 && !jobs) return p->fail(APSM_ERR_INVALID_ARGUMENT, "null job list");
    if (mode < 0 || mode > 2) return p->fail(APSM_ERR_INVALID_ARGUMENT, "unknown run mode");
    return p->run(lane, jobs, n_jobs, mode, true);
}

extern "C" apsm_status apsm_pool_autotune(apsm_pool* p, uint32_t lane, const apsm_job* jobs, uint32_t n_jobs,
                                          int mode, char* report, size_t report_len)
{
    if (!p) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(p->mu);
    if (lane >= p->lanes.size()) return p->fail(APSM_ERR_INVALID_ARGUMENT, "lane out of range");
    if (n_jobs == 0 || !jobs) return p->fail(APSM_ERR_INVALID_ARGUMENT, "autotune needs a batch");
    if (mode < 0 || mode > 2) return p->fail(APSM_ERR_INVALID_ARGUMENT, "unknown run mode");
    std::string rep;
    const apsm_status st = p->autotune(lane, jobs, n_jobs, mode, &rep);
    if (st == APSM_OK) copy_err(report, report_len, rep);
    return st;
}

extern "C" apsm_status apsm_pool_wait(apsm_pool* p, uint32_t lane)
{
    if (!p || lane >= p->lanes.size()) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(p->mu);
    return p->finish(lane);
}

extern "C" int apsm_pool_query(apsm_pool* p, uint32_t lane)
{
    if (!p || lane >= p->lanes.size()) return -int(APSM_ERR_INVALID_ARGUMENT);
    cudaError_t e = cudaEventQuery(p->lanes[lane].done);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) {
        cudaGetLastError();
        return 0;
    }
    p->cuda_fail(e, "cudaEventQuery");
    return -int(APSM_ERR_CUDA);
}

extern "C" void* apsm_pool_stream(apsm_pool* p, uint32_t lane)
{
    if (!p || lane >= p->lanes.size()) return nullptr;
    return (void*)p->lanes[lane].stream;
}

extern "C" uint64_t apsm_pool_job_bytes(const apsm_pool* p, const apsm_job* job)
{
    if (!p || !job || job->detector >= p->dets.size() || !p->dets[job->detector].live) return 0;
    const PoolDet& d = p->dets[job->detector];
    return job->kind == APSM_JOB_TRAIN ? p->train_bytes(d, job->length, true) : p->detect_bytes(d, job->length, true);
}

extern "C" apsm_status apsm_pool_check_job(const apsm_pool* p, const apsm_job* job)
{
    if (!p || !job) return APSM_ERR_INVALID_ARGUMENT;
    std::string msg;
    return p->job_error(*job, &msg);
}

extern "C" apsm_status apsm_pool_inject_fault(apsm_pool* p, int fault, uint32_t count)
{
    if (!p || fault != APSM_FAULT_LANE_ALLOC) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(p->mu);
    p->fault_lane_alloc = count;
    return APSM_OK;
}

extern "C" uint64_t apsm_pool_budget(const apsm_pool* p) { return p ? p->budget : 0; }

extern "C" uint64_t apsm_pool_bytes_in_use(const apsm_pool* p) { return p ? p->in_use() : 0; }

extern "C" apsm_status apsm_pool_last_ms(apsm_pool* p, uint32_t lane, float* train_ms, float* detect_ms)
{
    if (!p || lane >= p->lanes.size()) return APSM_ERR_INVALID_ARGUMENT;
    Lane& L = p->lanes[lane];
    cudaError_t e = cudaEventSynchronize(L.done);
    if (e != cudaSuccess) return p->cuda_fail(e, "cudaEventSynchronize");
    if (train_ms) {
        *train_ms = -1.f;
        if (L.have_train && cudaEventElapsedTime(train_ms, L.ev[0], L.ev[1]) != cudaSuccess) *train_ms = -1.f;
    }
    if (detect_ms) {
        *detect_ms = -1.f;
        if (L.have_detect && cudaEventElapsedTime(detect_ms, L.ev[2], L.ev[3]) != cudaSuccess) *detect_ms = -1.f;
    }
    cudaGetLastError();
    return APSM_OK;
}

extern "C" apsm_status apsm_pool_get_state(apsm_pool* p, uint32_t detector, uint32_t* rows, float* a, float* w)
{
    if (!p) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(p->mu);
    if (detector >= p->dets.size() || !p->dets[detector].live)
        return p->fail(APSM_ERR_INVALID_ARGUMENT, "unknown detector");
    for (auto& l : p->lanes) cudaStreamSynchronize(l.stream);
    const PoolDet& d = p->dets[detector];
    if (rows) *rows = d.used;
    if (a && d.used) {
        cudaError_t e = cudaMemcpy(a, d.a, sizeof(float) * d.used, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return p->cuda_fail(e, "cudaMemcpy(a)");
    }
    if (w) {
        cudaError_t e = cudaMemcpy(w, d.w, sizeof(float) * 2 * d.N, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return p->cuda_fail(e, "cudaMemcpy(w)");
    }
    return APSM_OK;
}

extern "C" int apsm_pool_last_launches(apsm_pool* p, uint32_t lane)
{
    if (!p || lane >= p->lanes.size()) return -1;
    return p->lanes[lane].launches;
}

extern "C" apsm_status apsm_pool_set_timing(apsm_pool* p, int on)
{
    if (!p) return APSM_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(p->mu);
    p->timing = on != 0;
    return APSM_OK;
}

extern "C" apsm_status apsm_pool_last_sweep_ms(apsm_pool* p, uint32_t lane, float* sweep_ms)
{
    if (!p || lane >= p->lanes.size() || !sweep_ms) return APSM_ERR_INVALID_ARGUMENT;
    Lane& L = p->lanes[lane];
    cudaError_t e = cudaEventSynchronize(L.done);
    if (e != cudaSuccess) return p->cuda_fail(e, "cudaEventSynchronize");
    *sweep_ms = -1.f;
    if (L.have_train && cudaEventElapsedTime(sweep_ms, L.ev[4], L.ev[5]) != cudaSuccess) *sweep_ms = -1.f;
    cudaGetLastError();
    return APSM_OK;
}
