// Host side of the B200 APSM detector: configuration (the reference factory's
// keys, defaults and validation), device state, the training schedule and the
// C ABI declared in include/apsm_b200.h.
#include "apsm_b200.h"
#include "apsm_kernels.cuh"
#include "apsm_host.hpp"
#include "json_lite.hpp"

#include <atomic>
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace apsm {

// ------------------------------------------------------------ config ------

static bool key_in(const std::string& k, std::initializer_list<const char*> keys)
{
    for (const char* v : keys)
        if (k == v) return true;
    return false;
}

static double num_value(const JsonValue& o, const char* key, double dflt)
{
    const JsonValue* v = o.find(key);
    if (!v) return dflt;
    if (v->kind != JsonValue::Number) throw std::invalid_argument(std::string("type_error: ") + key + " must be a number");
    return v->num;
}

static bool bool_value(const JsonValue& o, const char* key, bool dflt)
{
    const JsonValue* v = o.find(key);
    if (!v) return dflt;
    if (v->kind != JsonValue::Bool) throw std::invalid_argument(std::string("type_error: ") + key + " must be a boolean");
    return v->b;
}

static std::string str_value(const JsonValue& o, const char* key, const char* dflt)
{
    const JsonValue* v = o.find(key);
    if (!v) return dflt;
    if (v->kind != JsonValue::String) throw std::invalid_argument(std::string("type_error: ") + key + " must be a string");
    return v->str;
}

static uint32_t count_value(const JsonValue& o, const char* key, uint32_t dflt, uint32_t min_allowed)
{
    double v = num_value(o, key, dflt);
    if (!(v >= double(min_allowed)) || v > 1.0e9)
        throw std::invalid_argument(std::string("Invalid value for ") + key);
    return uint32_t(v);
}

// NomaDetectorFactory::build (noma_detector_factory.cu:57-65) and
// ApsmNomaDetectorFactory::build (apsm_noma_detector.cu:348-383).
Config parse_config(const std::string& json_text)
{
    JsonValue cfg = parse_json(json_text);
    if (cfg.kind != JsonValue::Object) throw std::invalid_argument("algorithm config must be a JSON object");
    Config c;
    const JsonValue* ot = cfg.find("otype");
    c.otype = (ot && ot->kind == JsonValue::String) ? ot->str : std::string(ot ? "<non-string>" : "null");
    // the reference iterates the keys in nlohmann's (sorted) order
    std::vector<std::string> keys;
    for (const auto& m : cfg.members) keys.push_back(m.first);
    std::sort(keys.begin(), keys.end());
    if (c.otype == "APSM") {
        for (const auto& k : keys)
            if (!key_in(k, {"otype", "llsInitialization", "trainingShuffle", "gaussianKernelWeight",
                            "gaussianKernelVariance", "windowSize", "sampleStep", "trainPasses",
                            "startWithFullWindow", "dictionarySize", "normConstraint", "eB", "detectVersion",
                            "trainVersion"}))
                throw std::invalid_argument("Invalid key: " + k);
        c.lls_init = bool_value(cfg, "llsInitialization", false);
        c.shuffle = bool_value(cfg, "trainingShuffle", false);
        c.wG = float(num_value(cfg, "gaussianKernelWeight", 0.5));
        c.wL = 1 - c.wG;
        c.variance = float(num_value(cfg, "gaussianKernelVariance", 0.05));
        c.window = count_value(cfg, "windowSize", 20, 1);
        c.step = count_value(cfg, "sampleStep", 2, 1);
        c.passes = count_value(cfg, "trainPasses", 1, 0);
        c.sfw = bool_value(cfg, "startWithFullWindow", false);
        c.dict_size = count_value(cfg, "dictionarySize", 685, 1);
        c.norm_constraint = float(num_value(cfg, "normConstraint", 0.));
        c.eB = float(num_value(cfg, "eB", 0.001));
        const std::string tv = str_value(cfg, "trainVersion", "exact");
        if (tv == "exact") c.train_incremental = false;
        else if (tv == "incremental") c.train_incremental = true;
        else throw std::invalid_argument("Unknown train version: " + tv);
        c.detect_version = str_value(cfg, "detectVersion", "balanced");
        if (c.detect_version == "original" || c.detect_version == "oldfast" || c.detect_version == "shmem" ||
            c.detect_version == "balanced")
            c.detect_mode = DetectMode::Exact;
        else if (c.detect_version == "gram_bf16") c.detect_mode = DetectMode::GramBF16;
        else if (c.detect_version == "gram_bf16x3") c.detect_mode = DetectMode::GramBF16x3;
        else if (c.detect_version == "gram_tf32") c.detect_mode = DetectMode::GramTF32;
        else if (c.detect_version == "gram_tf32x3") c.detect_mode = DetectMode::GramTF32x3;
        else throw std::invalid_argument("Unknown detect version: " + c.detect_version);
    } else if (c.otype == "LLS") {
        for (const auto& k : keys)
            if (k != "otype") throw std::invalid_argument("Invalid key: " + k);
    } else {
        throw std::invalid_argument("Unknown algorithm: " + c.otype);
    }
    return c;
}

// ------------------------------------------------------------ schedule ----

// The reference host step loop (apsm_train.cu:100-160) as a list of kernel
// steps over universe rows (rows present before the call, then the 2P new
// rows).  Returns the visible end after the sweep in *final_hi.
std::vector<TrainStep> build_schedule(const Config& c, uint32_t used_before, uint32_t P, uint32_t cap, int* final_hi)
{
    std::vector<TrainStep> steps;
    const uint32_t rows = 2 * P, q2 = 2 * c.window, s = c.step;
    uint32_t hi = used_before, next = 0;
    uint32_t last_hi = used_before;
    for (uint32_t pass = 0; pass < c.passes; ++pass) {
        if (pass == 0 && c.sfw) {
            uint32_t k = q2 > s ? q2 - s : 0;
            uint32_t r = std::min(k, rows - next);
            hi += r;
            next += r;
        }
        for (uint32_t sidx = c.sfw ? q2 : s; sidx <= rows; sidx += s) {
            if (pass == 0) {
                uint32_t r = std::min(s, rows - next);
                hi += r;
                next += r;
            }
            uint32_t n_launch = std::min(q2, sidx + (pass == 0 ? used_before : 0));
            uint32_t used_t = std::min(hi, cap);
            uint32_t wk = std::min(q2, used_t);
            uint32_t n_active = std::min(n_launch, wk);
            if (n_active == 0) continue;
            steps.push_back(TrainStep{int(hi), int(wk), int(n_active), int(last_hi)});
            last_hi = hi;
        }
    }
    *final_hi = int(hi);
    return steps;
}

// NomaDetector::shuffleData (noma_detector.cu:59-74): mt19937 seeded with
// {1,...,8}; rx rows and tx are shuffled with identical copies of the engine,
// i.e. by one permutation.  Returns perm with shuffled[i] = original[perm[i]].
std::vector<int> shuffle_permutation(uint32_t P)
{
    std::seed_seq seed{1, 2, 3, 4, 5, 6, 7, 8};
    std::mt19937 base(seed);
    std::vector<int> perm(P);
    for (uint32_t i = 0; i < P; ++i) perm[i] = int(i);
    std::mt19937 rng = base;
    std::shuffle(perm.begin(), perm.end(), rng);
    return perm;
}

} // namespace apsm

// ==================================================================== ABI ==

using namespace apsm;

static apsm_status fail(apsm_detector* h, apsm_status st, const std::string& msg)
{
    if (h) h->last_error = msg;
    return st;
}

static void copy_err(char* err, size_t errlen, const std::string& msg)
{
    if (err && errlen) {
        std::strncpy(err, msg.c_str(), errlen - 1);
        err[errlen - 1] = 0;
    }
}

extern "C" const char* apsm_version(void) { return "apsm_b200 0.1.0 (sm_100a)"; }

namespace {
std::atomic<unsigned long long> g_wait_limit_ns{2000000000ull};
}

unsigned long long apsm::wait_limit_ns() { return g_wait_limit_ns.load(std::memory_order_relaxed); }

extern "C" void apsm_set_wait_limit_ns(uint64_t ns) { g_wait_limit_ns.store(ns, std::memory_order_relaxed); }

extern "C" uint64_t apsm_wait_limit_ns(void) { return g_wait_limit_ns.load(std::memory_order_relaxed); }

extern "C" apsm_status apsm_create(const char* algorithm_json, uint32_t num_antennas, uint32_t num_users,
                                   apsm_detector** out, char* err, size_t errlen)
{
    if (!algorithm_json || !out) {
        copy_err(err, errlen, "null argument");
        return APSM_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    if (num_antennas == 0 || num_antennas > uint32_t(kMaxFeatures / 2)) {
        copy_err(err, errlen, "num_antennas must be in [1, " + std::to_string(kMaxFeatures / 2) + "]");
        return num_antennas == 0 ? APSM_ERR_INVALID_ARGUMENT : APSM_ERR_UNSUPPORTED;
    }
    if (num_users == 0) {
        copy_err(err, errlen, "num_users must be >= 1");
        return APSM_ERR_INVALID_ARGUMENT;
    }
    Config cfg;
    try {
        cfg = parse_config(algorithm_json);
    } catch (const std::exception& e) {
        copy_err(err, errlen, e.what());
        return APSM_ERR_INVALID_CONFIG;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        copy_err(err, errlen, "no CUDA device available");
        return APSM_ERR_NO_DEVICE;
    }
    auto* h = new apsm_detector();
    apsm_status st = h->init(cfg, num_antennas, num_users);
    if (st != APSM_OK) {
        copy_err(err, errlen, h->last_error);
        delete h;
        return st;
    }
    *out = h;
    return APSM_OK;
}

extern "C" void apsm_destroy(apsm_detector* h) { delete h; }

extern "C" const char* apsm_last_error(const apsm_detector* h) { return h ? h->last_error.c_str() : "null handle"; }

extern "C" void* apsm_stream(apsm_detector* h) { return h ? (void*)h->stream : nullptr; }

extern "C" apsm_status apsm_synchronize(apsm_detector* h)
{
    if (!h) return APSM_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(h, APSM_ERR_CUDA, cudaGetErrorString(e));
    return APSM_OK;
}

extern "C" apsm_status apsm_reset(apsm_detector* h)
{
    if (!h) return APSM_ERR_INVALID_ARGUMENT;
    return h->reset();
}

extern "C" uint32_t apsm_rows(const apsm_detector* h) { return h ? h->used : 0; }

extern "C" apsm_status apsm_train_device(apsm_detector* h, const float* d_rx, const float* d_tx, uint32_t P, void* stream)
{
    if (!h) return APSM_ERR_INVALID_ARGUMENT;
    if (!d_rx || !d_tx || P == 0) return fail(h, APSM_ERR_INVALID_ARGUMENT, "train: null buffer or P == 0");
    return h->train(reinterpret_cast<const float2*>(d_rx), reinterpret_cast<const float2*>(d_tx), P,
                    stream ? (cudaStream_t)stream : h->stream, nullptr);
}

extern "C" apsm_status apsm_detect_device(apsm_detector* h, const float* d_rx, uint32_t S, float* d_est, void* stream)
{
    if (!h) return APSM_ERR_INVALID_ARGUMENT;
    if (!d_rx || !d_est) return fail(h, APSM_ERR_INVALID_ARGUMENT, "detect: null buffer");
    if (S == 0) return APSM_OK;
    return h->detect(reinterpret_cast<const float2*>(d_rx), S, reinterpret_cast<float2*>(d_est),
                     stream ? (cudaStream_t)stream : h->stream);
}

extern "C" apsm_status apsm_train(apsm_detector* h, const float* rx, const float* tx, uint32_t P, float* ms)
{
    if (!h) return APSM_ERR_INVALID_ARGUMENT;
    if (!rx || !tx || P == 0) return fail(h, APSM_ERR_INVALID_ARGUMENT, "train: null buffer or P == 0");
    return h->train_host(reinterpret_cast<const float2*>(rx), reinterpret_cast<const float2*>(tx), P, ms);
}

extern "C" apsm_status apsm_train_history(apsm_detector* h, const float* rx, const float* tx, uint32_t P,
                                          const float* rx_val, const float* tx_val, uint32_t S,
                                          uint32_t bits_per_symbol, float modulation_scale, float* history,
                                          uint32_t max_steps, uint32_t* n_steps, float* ms)
{
    if (!h) return APSM_ERR_INVALID_ARGUMENT;
    if (n_steps) *n_steps = 0;
    if (!rx || !tx || P == 0) return fail(h, APSM_ERR_INVALID_ARGUMENT, "train: null buffer or P == 0");
    if (!rx_val || !tx_val || S == 0) return fail(h, APSM_ERR_INVALID_ARGUMENT, "train history: empty validation set");
    if (bits_per_symbol == 0 || bits_per_symbol > 16 || (bits_per_symbol > 1 && bits_per_symbol % 2) ||
        !(modulation_scale > 0.f))
        return fail(h, APSM_ERR_INVALID_ARGUMENT, "train history: invalid modulation (bits per symbol / scale)");
    if (!history && apsm_train_steps(h, P) > 0) return fail(h, APSM_ERR_INVALID_ARGUMENT, "train history: null output");
    return h->train_history_host(reinterpret_cast<const float2*>(rx), reinterpret_cast<const float2*>(tx), P,
                                 reinterpret_cast<const float2*>(rx_val), reinterpret_cast<const float2*>(tx_val), S,
                                 bits_per_symbol, modulation_scale, history, max_steps, n_steps, ms);
}

extern "C" uint32_t apsm_train_steps(const apsm_detector* h, uint32_t P) { return h ? h->train_steps(P) : 0; }

extern "C" apsm_status apsm_gaussian_variance(const apsm_detector* h, float* variance)
{
    if (!h || !variance) return APSM_ERR_INVALID_ARGUMENT;
    *variance = h->gaussian_variance();
    return APSM_OK;
}

extern "C" apsm_status apsm_norm_ratio(apsm_detector* h, uint32_t user, float* ratio)
{
    if (!h) return APSM_ERR_INVALID_ARGUMENT;
    if (!ratio) return fail(h, APSM_ERR_INVALID_ARGUMENT, "norm ratio: null output");
    return h->norm_ratio(user, ratio);
}

extern "C" apsm_status apsm_detect(apsm_detector* h, const float* rx, uint32_t S, float* est, float* ms)
{
    if (!h) return APSM_ERR_INVALID_ARGUMENT;
    if (!rx || !est) return fail(h, APSM_ERR_INVALID_ARGUMENT, "detect: null buffer");
    if (S == 0) {
        if (ms) *ms = 0.f;
        return APSM_OK;
    }
    return h->detect_host(reinterpret_cast<const float2*>(rx), S, reinterpret_cast<float2*>(est), ms);
}

extern "C" apsm_status apsm_get_state(apsm_detector* h, float* dict, float* a, float* w)
{
    if (!h) return APSM_ERR_INVALID_ARGUMENT;
    return h->get_state(dict, a, w);
}

extern "C" apsm_status apsm_copy_state(apsm_detector* dst, const apsm_detector* src)
{
    if (!dst || !src) return APSM_ERR_INVALID_ARGUMENT;
    if (dst == src) return APSM_OK;
    return dst->copy_state_from(*src);
}

extern "C" apsm_status apsm_last_kernel_ms(apsm_detector* h, float* sweep_ms, float* detect_ms)
{
    if (!h) return APSM_ERR_INVALID_ARGUMENT;
    return h->stage_ms(sweep_ms, detect_ms);
}
