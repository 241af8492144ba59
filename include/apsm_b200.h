/*
 * apsm_b200 — B200 (sm_100a) APSM multiuser detector, C ABI.
 *
 * This is the drop-in boundary for the reference's detector API
 * (fraunhoferhhi/libapsm, cpp/lib/noma/noma_detector.cuh:65-75).  All entry
 * points take plain pointers and sizes; no C++ or torch types cross it.
 *
 * Sample layout (identical to the reference's ComplexSampleMatrix /
 * ComplexSampleVector, cpp/lib/noma/types.cuh:95-100, flattened):
 *   rx  : num_antennas x n complex64, antenna-major:  rx[2*(a*n + i) + {0:re, 1:im}]
 *   tx  : P complex64 pilots per user, user-major for multi-user calls
 *   est : S complex64 estimates per user, user-major for multi-user calls
 *
 * Threading: a handle is not thread-safe (as the reference detector); distinct
 * handles may be used from distinct host threads.  Every call that takes host
 * buffers returns after the GPU work finished (the reference's calls are
 * synchronous too: CUDA_EventTimer::elapsed syncs, cpp/lib/cuda/cuda_eventtimer.cuh:121-128).
 * The library never calls exit(); every failure is a status code plus a message.
 */
#ifndef APSM_B200_H
#define APSM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    APSM_OK = 0,
    APSM_ERR_INVALID_ARGUMENT = 1, /* bad pointer / size / shape (reference: std::invalid_argument or assert) */
    APSM_ERR_INVALID_CONFIG = 2,   /* JSON config rejected (reference: std::invalid_argument from the factory) */
    APSM_ERR_CUDA = 3,             /* CUDA runtime error (reference: CUDA_CHECK prints and exits, cuda_errorhandling.cuh:98-108) */
    APSM_ERR_OUT_OF_MEMORY = 4,    /* device allocation failed or would exceed the handle's memory budget */
    APSM_ERR_UNSUPPORTED = 5,      /* valid config the B200 kernels do not implement (e.g. antenna count above the maximum) */
    APSM_ERR_NO_DEVICE = 6,        /* no usable sm_100 device */
    APSM_ERR_TIMEOUT = 7,          /* a host-side wait ran out of time */
    APSM_ERR_DEADLINE = 8,         /* a served request was not admitted into a batch by its deadline (dropped) */
    APSM_ERR_CANCELLED = 9         /* a served request was cancelled before it was admitted */
} apsm_status;

typedef struct apsm_detector apsm_detector;

/* Library version string and the device the handle runs on. */
const char* apsm_version(void);

/*
 * Create a detector from the reference's algorithm JSON object, e.g.
 *   {"otype":"APSM","windowSize":80,"gaussianKernelVariance":0.5,"eB":0.01}
 * Replaces NomaDetectorFactory::build (cpp/lib/noma/noma_detector_factory.cu:57-65)
 * and ApsmNomaDetectorFactory::build (cpp/lib/apsm/apsm_noma_detector.cu:348-383):
 * same keys, defaults and strict key check ("Invalid key: <k>",
 * "Unknown detect version: <v>", "Unknown algorithm: <otype>").
 * As the reference constructor does (apsm_noma_detector.cu:79-80), a non-zero
 * gaussianKernelVariance is multiplied by num_antennas^2.
 * Extensions (accepted in addition to the reference's keys):
 *   "detectVersion": "gram_bf16" | "gram_bf16x3" | "gram_tf32" | "gram_tf32x3"
 *        tensor-core Gram detection (tcgen05); the reference's four values
 *        ("original","oldfast","shmem","balanced") select the exact FP32 kernel.
 * num_users: detectors that share the same received signal (one per user of
 *   a cell, the reference CLI's -p mode, cpp/cli/detect/noma_detect.cpp:100-121);
 *   1 gives the reference's single-user NomaDetector.
 * err/errlen receive the message on failure (may be NULL/0).
 */
apsm_status apsm_create(const char* algorithm_json, uint32_t num_antennas, uint32_t num_users,
                        apsm_detector** out, char* err, size_t errlen);

/* Destroy the handle and free its device memory (reference dtor, apsm_noma_detector.cu:83-87). */
void apsm_destroy(apsm_detector* h);

/*
 * Online training on P pilots: NomaDetector::train (noma_detector.cuh:67;
 * apsm_noma_detector.cu:95-128 -> apsm_train.cu:80-166).
 * rx: N x P complex, tx: num_users x P complex.  Pilots append to the
 * detector's dictionary (capacity dictionarySize complex entries).
 * *ms (optional) receives the GPU time of the training work (CUDA events).
 */
apsm_status apsm_train(apsm_detector* h, const float* rx, const float* tx, uint32_t P, float* ms);

/*
 * Training with a per-step history: NomaDetector::train with a NomaValSet
 * (noma_detector.cuh:69, noma_train_history.cuh:64-99; recorded by
 * apsm_train.cu:147-156, computed as noma_train_history.cu:65-248).  Trains
 * exactly like apsm_train and, for the model after every step, records EVM,
 * SER and BER of this call's training symbols and of the validation set
 * rx_val (N x S complex) / tx_val (num_users x S complex, S > 0).
 * history: num_users x steps x 6 floats, per step train EVM, SER, BER,
 * validation EVM, SER, BER; steps = apsm_train_steps(h, P), which must be
 * <= max_steps (else APSM_ERR_INVALID_ARGUMENT before any work).
 * bits_per_symbol / modulation_scale: Modulation::getBitPerSymbol / getScale
 * of the symbols (the reference's NomaTrainHistory constructor arguments).
 * An LLS detector trains and records nothing (*n_steps = 0), as the
 * reference's LLS detector ignores the validation set (lls_detector.cu:136).
 */
apsm_status apsm_train_history(apsm_detector* h, const float* rx, const float* tx, uint32_t P, const float* rx_val,
                               const float* tx_val, uint32_t S, uint32_t bits_per_symbol, float modulation_scale,
                               float* history, uint32_t max_steps, uint32_t* n_steps, float* ms);

/*
 * The effective Gaussian variance of the model (apsm_parameters::
 * gaussianKernelVariance after the constructor's N^2 scaling,
 * apsm_noma_detector.cu:79-80, or, for a configured 0, the heuristic's value
 * once training ran: computeGaussianVarianceHeuristic, :193-218, which the
 * reference prints).  0 before a heuristic detector's first training call.
 */
apsm_status apsm_gaussian_variance(const apsm_detector* h, float* variance);

/*
 * ApsmNomaDetector::computeNormRatio (apsm_noma_detector.cu:220-311): the
 * ratio wL |w|^2 / (wG sum_ij a_i a_j k(d_i, d_j)) of the linear to the
 * Gaussian share of user `user`'s model, over the current dictionary.
 * APSM detectors only (APSM_ERR_UNSUPPORTED for LLS).  Synchronous.
 */
apsm_status apsm_norm_ratio(apsm_detector* h, uint32_t user, float* ratio);

/* Training steps (history rows per user) a train call with P pilots runs on
 * the detector's current state; 0 for LLS detectors.  No reference
 * counterpart (its history vectors grow as they are filled). */
uint32_t apsm_train_steps(const apsm_detector* h, uint32_t P);

/*
 * Detection of S data symbols: NomaDetector::detect (noma_detector.cuh:70;
 * apsm_noma_detector.cu:130-143 -> apsm_detect.cu:948-992).
 * rx: N x S complex, est: num_users x S complex (written).
 */
apsm_status apsm_detect(apsm_detector* h, const float* rx, uint32_t S, float* est, float* ms);

/* NomaDetector::resetState (noma_detector.cuh:73; apsm_noma_detector.cu:89-93). */
apsm_status apsm_reset(apsm_detector* h);

/*
 * Device-resident variants: the same work on buffers already in HBM, enqueued
 * on `stream` (a cudaStream_t, NULL = the handle's own stream) without a host
 * synchronisation.  Layouts as above.  No counterpart in the reference (its
 * train/detect always copy host vectors in, cuda_matrix_host.cu:105-149).
 */
apsm_status apsm_train_device(apsm_detector* h, const float* d_rx, const float* d_tx, uint32_t P, void* stream);
apsm_status apsm_detect_device(apsm_detector* h, const float* d_rx, uint32_t S, float* d_est, void* stream);

/*
 * Detection that allocates no device memory: the exact FP32 detection of
 * apsm_detect_device, with the packed data rows in a fixed 8 MiB device array
 * of the library instead of a buffer of the handle that grows with S.  For
 * callers that must not allocate on the call path.  No counterpart in the
 * reference (its detect allocates and copies per call, cuda_matrix_host.cu:105-149).
 * Limit: 2 * S * Dp * 4 bytes <= 8 MiB, Dp = 2N rounded up to 4 (S <= 32768
 * at N = 16); larger S returns APSM_ERR_INVALID_ARGUMENT.  APSM handles with
 * the reference's detectVersion values only (else APSM_ERR_UNSUPPORTED).  The
 * first call on a device looks up the array's address (make it before any
 * stream capture); the array is shared by all handles on the device, so calls
 * that overlap on a device race and must be serialised by the caller.  The
 * looked-up address is kept for the life of the process: cudaDeviceReset on a
 * device that has used this entry point is not supported (the library's
 * module would load again, possibly at another address).
 */
apsm_status apsm_detect_device_noalloc(apsm_detector* h, const float* d_rx, uint32_t S, float* d_est, void* stream);

/* The handle's CUDA stream (cudaStream_t) and a blocking wait on it. */
void* apsm_stream(apsm_detector* h);
apsm_status apsm_synchronize(apsm_detector* h);

/*
 * Model snapshot (reference: getTrainingState, apsm_noma_detector.cuh:93):
 * rows = 2 x (complex dictionary entries in use); dict rows x 2N (Dedup real
 * rows, oldest first), a: num_users x rows, w: num_users x 2N.  Any pointer may
 * be NULL.  apsm_rows returns the current row count.
 */
uint32_t apsm_rows(const apsm_detector* h);
apsm_status apsm_get_state(apsm_detector* h, float* dict, float* a, float* w);

/*
 * Copies the whole trained state of src (dictionary rows, their targets and
 * coefficients, linear weights, the kernel variance a heuristic chose) into
 * dst, on the device.  Both are APSM detectors on one device with the same
 * antennas, users, dictionarySize and kernel weights; dst's configured
 * gaussianKernelVariance must be 0 (heuristic) or equal src's.  dst's
 * detection form (detectVersion) is its own, so one trained model can be
 * evaluated in several precisions.  Waits for src's stream; the copies are
 * ordered on dst's stream.  No reference counterpart (the reference's detector
 * state is private, apsm_noma_detector.cuh:93 only reads it).
 */
apsm_status apsm_copy_state(apsm_detector* dst, const apsm_detector* src);

/*
 * GPU time (CUDA events, ms) of the last training sweep kernel and of the last
 * detection kernel of this handle; -1 when that stage has not run.  Blocks
 * until those kernels finished.  Replaces nothing in the reference (its
 * train/detect return one event time each, apsm_train.cu:163-165,
 * apsm_detect.cu:972-974); used for roofline accounting.
 */
apsm_status apsm_last_kernel_ms(apsm_detector* h, float* sweep_ms, float* detect_ms);

/* Last error message of the handle ("" if none). */
const char* apsm_last_error(const apsm_detector* h);

/* Limit of the bounded waits inside the tensor-core detection kernels
 * (nanoseconds, process-wide; 2 s by default).  No counterpart in the
 * reference, whose CUDA errors end the process (CUDA_CHECK,
 * cpp/lib/cuda/cuda_errorhandling.cuh:98-108).  A kernel whose wait expires
 * stops its work, still waits for its own copies and tensor-core products,
 * releases tensor memory and flags the call, which returns APSM_ERR_CUDA; the
 * handle stays usable.  0 makes every wait that is not already complete give
 * up at once: a way to test the expiry path.  Launches read the value when
 * they are issued. */
void apsm_set_wait_limit_ns(uint64_t ns);
uint64_t apsm_wait_limit_ns(void);

/* Measured exponential throughput of the current device's SFUs
 * (ex2.approx.ftz.f32 per second, all SMs; the detection kernels' every
 * exponential is one such instruction): the denominator of the detection
 * stage's roofline.  Runs a warm-up and a timed launch of ~2 ms on its own
 * stream; ms (optional) receives the timed launch's duration.  No counterpart
 * in the reference. */
apsm_status apsm_measure_ex2_rate(double* per_second, float* ms);

/* ======================================================================
 * Detector pool: many resident detectors (users x cells), batched jobs.
 *
 * The reference runs one ApsmNomaDetector per user, each with its own
 * stream, host thread and calls (its CLI's -p mode, noma_detect.cpp:109-112;
 * one train/detect per detector, noma_detector.cuh:65-75).  A pool holds the
 * device state of many detectors of one algorithm config (each with its own
 * antenna count) and runs a batch of their train/detect calls in a handful
 * of launches: every training job of the batch in one persistent sweep
 * launch, every detection job in one launch per antenna class.  Per detector
 * the semantics are those of NomaDetector::train / detect; results equal the
 * single-detector path within the FP32 tolerance (1e-4 relative).
 *
 * Restrictions: otype "APSM" without llsInitialization or normConstraint,
 * gaussianKernelVariance > 0, even sampleStep <= 8, dictionarySize >=
 * windowSize + sampleStep / 2, N <= 64 antennas.
 * ==================================================================== */
typedef struct apsm_pool apsm_pool;

typedef enum { APSM_JOB_TRAIN = 0, APSM_JOB_DETECT = 1 } apsm_job_kind;

/* Train-job flag: reset the detector (resetState, apsm_noma_detector.cu:89-93)
 * before training on this job's pilots. */
#define APSM_JOB_FRESH 1u

typedef struct {
    uint32_t detector; /* id from apsm_pool_add */
    uint32_t kind;     /* apsm_job_kind */
    uint32_t length;   /* pilots P (train) or data symbols S (detect) */
    uint32_t flags;    /* APSM_JOB_FRESH or 0 */
    const float* rx;   /* N x length complex64, antenna-major (NomaDetector's rxSig[N][length]) */
    const float* tx;   /* train: length complex64 pilots of this detector's user; detect: NULL */
    float* est;        /* detect: length complex64 soft estimates (output); train: NULL */
} apsm_job;

/* A pool for one algorithm config.  hbm_budget_bytes bounds the device memory
 * of resident detector state plus batch scratch (0: no bound).  lanes >= 1
 * independent streams, each with its own scratch, so batches can overlap. */
apsm_status apsm_pool_create(const char* algorithm_json, uint64_t hbm_budget_bytes, uint32_t lanes,
                             apsm_pool** out, char* err, size_t errlen);
void apsm_pool_destroy(apsm_pool* p);

/* Resident detector with num_antennas antennas (fresh state, like resetState);
 * APSM_ERR_OUT_OF_MEMORY if its state does not fit the budget. */
apsm_status apsm_pool_add(apsm_pool* p, uint32_t num_antennas, uint32_t* detector);
apsm_status apsm_pool_remove(apsm_pool* p, uint32_t detector);
apsm_status apsm_pool_reset(apsm_pool* p, uint32_t detector);

/* Run modes of apsm_pool_run. */
#define APSM_RUN_HOST 0       /* host buffers; returns when the estimates are written */
#define APSM_RUN_DEVICE 1     /* device buffers; returns once enqueued on the lane's stream */
#define APSM_RUN_HOST_ASYNC 2 /* host buffers; returns once enqueued, estimates arrive with apsm_pool_wait */

/* Runs a batch on a lane: all training jobs first (in one sweep launch; a
 * detector may be trained at most once per batch), then all detection jobs,
 * which see this batch's training.  Host modes, inputs: a batch with 4 MB or
 * more of training inputs whose buffers are page-locked and mapped for the
 * device has them read in place by the packing kernel (one launch per antenna
 * class on a second stream, beside the kernel columns of the classes packed
 * before); detection samples in page-locked buffers are copied to the device
 * straight from them on that stream while the batch trains; in a batch that
 * trains and has 4 MB or more of detection samples in pageable buffers, those
 * are staged by host helper threads and uploaded on that stream in groups of
 * about 32 MB while the batch trains (the call returns once they are staged);
 * everything else (small batches, training inputs in pageable buffers) is
 * staged through the lane's pinned buffer and uploaded with the job
 * descriptors.  Detection runs in segments of one launch shape, each waiting
 * for its own samples only.  Estimates: into page-locked,
 * device-mapped caller buffers (batches with 4 MB of estimates or more) the
 * detection kernels write them in place, so such buffers hold partial
 * estimates while the batch runs; otherwise each launch's estimates come
 * back in one device-to-host copy and are scattered to the callers' buffers
 * when the batch is finished.  The caller keeps its buffers alive until the
 * batch finished.  A later run (or reserve / autotune) on the lane finishes
 * a lane's pending APSM_RUN_HOST_ASYNC batch first and returns its status if
 * it failed.  A detector must not be in batches on two lanes at once. */
apsm_status apsm_pool_run(apsm_pool* p, uint32_t lane, const apsm_job* jobs, uint32_t n_jobs, int mode);
/* Waits for the lane's last batch and, for APSM_RUN_HOST_ASYNC, writes its
 * estimates to the caller's buffers; returns the batch's status (an expired
 * bounded wait of a tensor-core kernel: APSM_ERR_CUDA). */
apsm_status apsm_pool_wait(apsm_pool* p, uint32_t lane);

/*
 * Grows the lane's device scratch and page-locked buffers to what this batch
 * (same arguments as apsm_pool_run) needs, without running it or changing any
 * detector; returns once the memory is in place.  A pending
 * APSM_RUN_HOST_ASYNC batch of the lane is finished first (its estimates are
 * written, its failure is returned): growth retires the buffers it reads.  A lane grows its buffers on
 * demand otherwise, and growing them (mapping device memory, page-locking
 * host memory) stalls the batch that needs it for milliseconds: a request
 * server reserves every lane for its largest batch before taking requests.
 * No reference counterpart.
 */
apsm_status apsm_pool_reserve(apsm_pool* p, uint32_t lane, const apsm_job* jobs, uint32_t n_jobs, int mode);

/*
 * Launch-shape autotuner: runs the batch (same arguments as apsm_pool_run;
 * it is waited for) once per candidate of each launch shape it exercises --
 * training-sweep CTAs per SM, tensor-core detection pipeline stages, CUDA-core
 * detection split threshold -- keeps the fastest by GPU time, and uses it for
 * every later batch of this pool.  The detectors the batch trains get their
 * state back: the call changes no detector and no result.  report (may be
 * NULL) receives a JSON object with the trials and the chosen shape.  No
 * reference counterpart (the reference launches fixed shapes).
 */
apsm_status apsm_pool_autotune(apsm_pool* p, uint32_t lane, const apsm_job* jobs, uint32_t n_jobs, int mode,
                               char* report, size_t report_len);
/* 1 when the lane's GPU work finished (call apsm_pool_wait for the estimates
 * of an asynchronous host batch), 0 while it runs, < 0 on error. */
int apsm_pool_query(apsm_pool* p, uint32_t lane);
void* apsm_pool_stream(apsm_pool* p, uint32_t lane);

/* Device scratch bytes the job needs in a batch (admission by HBM budget),
 * the pool's budget and the bytes currently held (resident + scratch). */
uint64_t apsm_pool_job_bytes(const apsm_pool* p, const apsm_job* job);
uint64_t apsm_pool_budget(const apsm_pool* p);
uint64_t apsm_pool_bytes_in_use(const apsm_pool* p);

/* GPU time (ms, CUDA events) of the lane's last batch: training (kernel
 * columns + sweep) and detection stages; blocks until the batch finished. */
apsm_status apsm_pool_last_ms(apsm_pool* p, uint32_t lane, float* train_ms, float* detect_ms);

/* Per-stage GPU events of every batch (default on): apsm_pool_last_ms and
 * apsm_pool_last_sweep_ms report -1 while off.  Off saves six event records
 * per batch on the latency-critical path (the request server turns it off).
 * No reference counterpart. */
apsm_status apsm_pool_set_timing(apsm_pool* pool, int on);

/* GPU time (ms) of the persistent training sweep kernel of the lane's last batch (-1: none). */
apsm_status apsm_pool_last_sweep_ms(apsm_pool* p, uint32_t lane, float* sweep_ms);

/* Kernels the lane's last batch launched (its own kernels; memsets and copies excluded). */
int apsm_pool_last_launches(apsm_pool* p, uint32_t lane);

/* The checks apsm_pool_run applies to one job on its own: known detector and
 * kind, buffers present (APSM_ERR_INVALID_ARGUMENT otherwise).  Reads the
 * detector table without locking: not concurrently with apsm_pool_add /
 * apsm_pool_remove.  No counterpart in the reference. */
apsm_status apsm_pool_check_job(const apsm_pool* p, const apsm_job* job);

/* Host-side fault injection, for tests of the failure paths (no counterpart in
 * the reference, whose CUDA errors end the process).  APSM_FAULT_LANE_ALLOC:
 * the pool's next `count` lane-scratch growths fail as an allocation would
 * (the batch returns APSM_ERR_OUT_OF_MEMORY; the lane grows again on a later
 * batch).  APSM_FAULT_DROP_REQUEST (server): the next `count` submitted
 * requests are lost on their way into the queue; they end only by their
 * deadline (APSM_ERR_DEADLINE) or apsm_server_cancel.  Nothing faults the GPU. */
typedef enum { APSM_FAULT_LANE_ALLOC = 1, APSM_FAULT_DROP_REQUEST = 2 } apsm_fault;
apsm_status apsm_pool_inject_fault(apsm_pool* p, int fault, uint32_t count);

/* Snapshot of a detector: rows in use, a (rows), w (2N); pointers may be NULL. */
apsm_status apsm_pool_get_state(apsm_pool* p, uint32_t detector, uint32_t* rows, float* a, float* w);
const char* apsm_pool_last_error(const apsm_pool* p);

/* ======================================================================
 * Request server: continuous batching of per-TTI requests over a pool.
 *
 * No counterpart in the reference (its CLI processes one frame per detector
 * and thread, noma_detect.cpp:100-137).  A worker thread admits waiting
 * requests into batches on the pool's first `lanes` lanes as they become
 * free: per detector, requests keep their arrival order and a detector with
 * a batch in flight waits; a batch is bounded by max_batch requests and by
 * the device scratch the pool's HBM budget leaves per lane.  Batches on
 * different lanes overlap on the GPU.  Every request is one apsm_job with
 * host buffers that stay valid until the request finished.  A request's
 * result is the same whichever requests share its batch.  The pool must not
 * be used directly while a server runs on it.
 * ==================================================================== */
typedef struct apsm_server apsm_server;

apsm_status apsm_server_create(apsm_pool* pool, uint32_t lanes, uint32_t max_batch, apsm_server** out);
/* Finishes every queued request, then stops the worker. */
void apsm_server_destroy(apsm_server* s);
/* Queues a request (deadline: the server's default).  A malformed request
 * (apsm_pool_check_job) or one whose scratch alone exceeds the pool's HBM
 * budget is rejected here (APSM_ERR_INVALID_ARGUMENT / APSM_ERR_OUT_OF_MEMORY,
 * no ticket), so it cannot fail the batch it would join. */
apsm_status apsm_server_submit(apsm_server* s, const apsm_job* job, uint64_t* ticket);
/* As apsm_server_submit, with a deadline deadline_s seconds after submission
 * (0: none; < 0: the server's default).  A request not admitted into a batch
 * by its deadline ends with APSM_ERR_DEADLINE without running; one admitted
 * in time runs to completion (its completion time, apsm_server_times, may be
 * later than the deadline).  A dropped training request leaves the detector's
 * state as it was; the detector's later requests proceed. */
apsm_status apsm_server_submit_deadline(apsm_server* s, const apsm_job* job, double deadline_s, uint64_t* ticket);
/* Default deadline (seconds after submission, 0: none) of later submissions. */
apsm_status apsm_server_set_deadline(apsm_server* s, double seconds);
/* Ends a request that is not admitted yet with APSM_ERR_CANCELLED.  A request
 * already on the GPU runs to completion (APSM_ERR_UNSUPPORTED); a finished or
 * unknown one: APSM_ERR_INVALID_ARGUMENT. */
apsm_status apsm_server_cancel(apsm_server* s, uint64_t ticket);
/* Requests dropped at their deadline, cancelled, and rejected at submission. */
apsm_status apsm_server_counts(apsm_server* s, uint64_t* dropped, uint64_t* cancelled, uint64_t* rejected);
/* See apsm_pool_inject_fault (APSM_FAULT_DROP_REQUEST). */
apsm_status apsm_server_inject_fault(apsm_server* s, int fault, uint32_t count);
/* 1 when the request finished (*status its result), 0 while pending, -1 unknown ticket. */
int apsm_server_poll(apsm_server* s, uint64_t ticket, apsm_status* status);
/* Blocks until the request finished (its status) or timeout_s passed (APSM_ERR_TIMEOUT). */
apsm_status apsm_server_wait(apsm_server* s, uint64_t ticket, double timeout_s);
/* Host times (seconds, apsm_server_clock) of submission, admission into a batch, completion. */
apsm_status apsm_server_times(apsm_server* s, uint64_t ticket, double* submit_s, double* start_s, double* done_s);
/* Forget a finished request. */
apsm_status apsm_server_release(apsm_server* s, uint64_t ticket);
/* Batches launched and requests they held. */
apsm_status apsm_server_stats(apsm_server* s, uint64_t* batches, uint64_t* jobs);
/* The monotonic clock of the request times, in seconds. */
double apsm_server_clock(void);

#ifdef __cplusplus
}
#endif
#endif /* APSM_B200_H */
