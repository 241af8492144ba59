// TEST INFRASTRUCTURE ONLY — not part of the product.
//
// C-ABI shim over the *reference* libapsm library compiled from its own
// sources (see oracle/Makefile).  It lets the parity tests and the golden
// fixture generator drive the reference's public C++ detector API
// (NomaDetectorFactory::build -> NomaDetector::train / detect,
// cpp/lib/noma/noma_detector_factory.cu:57-65, cpp/lib/noma/noma_detector.cuh:65-75)
// on the same inputs as the B200 detector.  Only tests/ and the fixture
// script may load the resulting library.
//
// Sample layout at this boundary (same as the product C-ABI):
//   rx  : antenna-major complex64, rx[a * samples + n] = (re, im)
//   tx  : complex64 per pilot
//   est : complex64 per data symbol

#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>
#include <nlohmann/json.hpp>

#include "noma/noma_detector_factory.cuh"
#include "noma/noma_train_history.cuh"
#include "apsm/apsm_versions.cuh"
#include "apsm/apsm_noma_detector.cuh"

namespace {

ComplexSampleMatrix to_matrix(const float* rx, uint32_t n_ant, uint32_t n)
{
    ComplexSampleMatrix m(n_ant, ComplexSampleVector(n));
    for (uint32_t a = 0; a < n_ant; ++a)
        for (uint32_t i = 0; i < n; ++i)
            m[a][i] = ComplexSample(rx[2 * (size_t(a) * n + i)], rx[2 * (size_t(a) * n + i) + 1]);
    return m;
}

ComplexSampleVector to_vector(const float* v, uint32_t n)
{
    ComplexSampleVector out(n);
    for (uint32_t i = 0; i < n; ++i)
        out[i] = ComplexSample(v[2 * i], v[2 * i + 1]);
    return out;
}

void set_err(char* err, size_t errlen, const std::string& msg)
{
    if (err && errlen) {
        std::strncpy(err, msg.c_str(), errlen - 1);
        err[errlen - 1] = 0;
    }
}

} // namespace

extern "C" {

struct ref_handle {
    std::unique_ptr<NomaDetector> det;
};

int ref_create(const char* algorithm_json, uint32_t n_ant, ref_handle** out, char* err, size_t errlen)
{
    try {
        auto cfg = nlohmann::json::parse(algorithm_json);
        auto* h = new ref_handle;
        h->det = NomaDetectorFactory::build(cfg, n_ant);
        *out = h;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return 1;
    }
}

int ref_train(ref_handle* h, const float* rx, const float* tx, uint32_t n_ant, uint32_t P, float* ms)
{
    float t = h->det->train(to_matrix(rx, n_ant, P), to_vector(tx, P));
    if (ms) *ms = t;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

int ref_detect(ref_handle* h, const float* rx, uint32_t n_ant, uint32_t S, float* est, float* ms)
{
    ComplexSampleVector out;
    float t = h->det->detect(to_matrix(rx, n_ant, S), out);
    if (ms) *ms = t;
    if (out.size() != S) return 3;
    std::memcpy(est, out.data(), sizeof(float) * 2 * S);
    return 0;
}

// NomaDetector::train with a validation set (NomaValSet, cpp/lib/noma/noma_train_history.cuh:99;
// used so by the reference CLI, cpp/cli/detect/noma_detect.cpp:124-145).  out: max_steps x 6 =
// train EVM, SER, BER, validation EVM, SER, BER per recorded step; *n_steps = steps recorded.
int ref_train_history(ref_handle* h, const float* rx, const float* tx, uint32_t n_ant, uint32_t P,
                      const float* rx_val, const float* tx_val, uint32_t S, uint32_t bps, float mod_scale,
                      float* out, uint32_t max_steps, uint32_t* n_steps, float* ms)
{
    NomaTrainHistory stats(bps, mod_scale);
    const ComplexSampleMatrix rxv = to_matrix(rx_val, n_ant, S);
    const ComplexSampleVector txv = to_vector(tx_val, S);
    NomaValSet vs;
    vs.emplace(std::make_tuple(std::ref(stats), std::cref(rxv), std::cref(txv)));
    float t = h->det->train(to_matrix(rx, n_ant, P), to_vector(tx, P), vs);
    if (ms) *ms = t;
    if (cudaDeviceSynchronize() != cudaSuccess) return 2;
    const size_t n = stats.evmTrain.size();
    if (n_steps) *n_steps = uint32_t(n);
    for (size_t i = 0; i < n && i < max_steps; ++i) {
        const float row[6] = {stats.evmTrain[i], stats.serTrain[i], stats.berTrain[i],
                              stats.evmVal[i],   stats.serVal[i],   stats.berVal[i]};
        std::memcpy(out + 6 * i, row, sizeof(row));
    }
    return n > max_steps ? 3 : 0;
}

// ApsmNomaDetector::computeNormRatio (apsm_noma_detector.cuh:92), whichever detect version
// the factory built.
int ref_norm_ratio(ref_handle* h, float* out)
{
    NomaDetector* d = h->det.get();
    if (auto* x = dynamic_cast<ApsmNomaDetector<apsm_versions::APSM_DETECT_BALANCED>*>(d)) *out = x->computeNormRatio();
    else if (auto* x = dynamic_cast<ApsmNomaDetector<apsm_versions::APSM_DETECT_ORIGINAL>*>(d)) *out = x->computeNormRatio();
    else if (auto* x = dynamic_cast<ApsmNomaDetector<apsm_versions::APSM_DETECT_OLDFAST>*>(d)) *out = x->computeNormRatio();
    else if (auto* x = dynamic_cast<ApsmNomaDetector<apsm_versions::APSM_DETECT_SHMEM>*>(d)) *out = x->computeNormRatio();
    else return 1;
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

void ref_reset(ref_handle* h) { h->det->resetState(); }

void ref_destroy(ref_handle* h) { delete h; }

// The reference CLI's "-p" mode (cpp/cli/detect/noma_detect.cpp:100-121):
// one detector per user, each on its own host thread (and its own stream),
// all trained on the same rx pilots and detecting the same rx data.
// tx: n_users x P complex, est: n_users x S complex.
int ref_run_users_threaded(const char* algorithm_json, uint32_t n_ant, uint32_t n_users,
                           const float* rx_train, const float* tx, uint32_t P,
                           const float* rx_data, uint32_t S, float* est, char* err, size_t errlen)
{
    try {
        auto cfg = nlohmann::json::parse(algorithm_json);
        ComplexSampleMatrix rxt = to_matrix(rx_train, n_ant, P);
        ComplexSampleMatrix rxd = to_matrix(rx_data, n_ant, S);
        std::vector<std::unique_ptr<NomaDetector>> dets;
        std::vector<ComplexSampleVector> outs(n_users);
        std::vector<ComplexSampleVector> txs;
        for (uint32_t u = 0; u < n_users; ++u) {
            dets.push_back(NomaDetectorFactory::build(cfg, n_ant));
            txs.push_back(to_vector(tx + 2 * size_t(u) * P, P));
        }
        std::vector<std::thread> threads;
        for (uint32_t u = 0; u < n_users; ++u)
            threads.emplace_back([&, u]() {
                dets[u]->train(rxt, txs[u]);
                dets[u]->detect(rxd, outs[u]);
            });
        for (auto& t : threads) t.join();
        if (cudaDeviceSynchronize() != cudaSuccess) return 2;
        for (uint32_t u = 0; u < n_users; ++u) {
            if (outs[u].size() != S) return 3;
            std::memcpy(est + 2 * size_t(u) * S, outs[u].data(), sizeof(float) * 2 * S);
        }
        return 0;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return 1;
    }
}

} // extern "C"
