// apsm_b200 — C++ drop-in for the reference's detector API, header-only over
// the C ABI of apsm_b200.h.
//
// Mirrors fraunhoferhhi/libapsm:
//   class NomaDetector            cpp/lib/noma/noma_detector.cuh:65-75
//   NomaDetectorFactory::build    cpp/lib/noma/noma_detector_factory.cu:57-65
//   NomaTrainHistory, NomaValSet  cpp/lib/noma/noma_train_history.cuh:64-99
//   sample typedefs               cpp/lib/noma/types.cuh:69-100
// Same signatures and semantics: train/detect return the GPU time in ms,
// detect resizes estData, configuration errors throw std::invalid_argument
// (as the reference factories do), other failures throw std::runtime_error
// (the reference prints and exits instead).  Any JSON type with a dump()
// method (nlohmann::json included) can be passed to the factory.
#pragma once

#include "apsm_b200.h"

#include <complex>
#include <cstdint>
#include <fstream>
#include <functional>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

namespace apsm_b200 {

typedef float RealSample;
typedef std::vector<RealSample> RealSampleVector;
typedef std::vector<RealSampleVector> RealSampleMatrix;
typedef std::complex<RealSample> ComplexSample;
typedef std::vector<ComplexSample> ComplexSampleVector;
typedef std::vector<ComplexSampleVector> ComplexSampleMatrix;

// Per-step metrics of a training call with a validation set: after every
// training step EVM, SER and BER of the training symbols and of the
// validation set under that step's model (computed on the GPU by
// apsm_train_history).  toCsv writes the reference's CSV
// (noma_train_history.cu:237-248).
class NomaTrainHistory {
public:
    NomaTrainHistory(uint32_t bitPerSymbol, float modulationScale)
        : bitPerSymbol(bitPerSymbol), modulationScale(modulationScale)
    {
    }
    NomaTrainHistory() = delete;
    NomaTrainHistory(const NomaTrainHistory&) = delete;
    NomaTrainHistory& operator=(const NomaTrainHistory&) = delete;

    void toCsv(const std::string& filename) const
    {
        std::ofstream file(filename, std::ios::out | std::ios::trunc);
        file << "step,train_evm,train_ser,train_ber,val_evm,val_ser,val_ber" << std::endl;
        for (size_t i = 0; i < evmTrain.size(); ++i) {
            file << i << "," << evmTrain[i] << "," << serTrain[i] << "," << berTrain[i] << ",";
            file << evmVal[i] << "," << serVal[i] << "," << berVal[i] << std::endl;
        }
    }

    RealSampleVector evmTrain, evmVal, serTrain, serVal, berTrain, berVal;
    const uint32_t bitPerSymbol;
    const float modulationScale;
};

typedef std::optional<std::tuple<NomaTrainHistory&, const ComplexSampleMatrix&, const ComplexSampleVector&>> NomaValSet;

class NomaDetector {
public:
    virtual ~NomaDetector() {}
    virtual float train(const ComplexSampleMatrix& rxSigTraining, const ComplexSampleVector& txSigTraining,
                        NomaValSet valSet = std::nullopt) = 0;
    virtual float detect(const ComplexSampleMatrix& rxSigData, ComplexSampleVector& estData) = 0;
    virtual void resetState() = 0;
};

namespace detail {

inline void throw_status(apsm_status st, const std::string& msg)
{
    if (st == APSM_OK) return;
    if (st == APSM_ERR_INVALID_CONFIG || st == APSM_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// antenna-major complex matrix -> contiguous N x n complex64
inline std::vector<ComplexSample> flatten(const ComplexSampleMatrix& m, uint32_t rows, size_t* n)
{
    if (m.size() != rows) throw std::invalid_argument("sample matrix has " + std::to_string(m.size()) +
                                                      " antenna rows, detector expects " + std::to_string(rows));
    *n = rows ? m[0].size() : 0;
    std::vector<ComplexSample> flat;
    flat.reserve(rows * *n);
    for (const auto& r : m) {
        if (r.size() != *n) throw std::invalid_argument("ragged sample matrix");
        flat.insert(flat.end(), r.begin(), r.end());
    }
    return flat;
}

} // namespace detail

// One detector (or, with numUsers > 1, the detectors of several users that
// share the received signal).  Not thread-safe; one instance per host thread.
class ApsmB200Detector : public NomaDetector {
public:
    ApsmB200Detector(const std::string& algorithmJson, uint32_t numAntennas, uint32_t numUsers = 1)
        : numAntennas_(numAntennas), numUsers_(numUsers)
    {
        char err[512] = {0};
        apsm_status st = apsm_create(algorithmJson.c_str(), numAntennas, numUsers, &h_, err, sizeof(err));
        detail::throw_status(st, err);
    }
    ~ApsmB200Detector() override { apsm_destroy(h_); }
    ApsmB200Detector(const ApsmB200Detector&) = delete;
    ApsmB200Detector& operator=(const ApsmB200Detector&) = delete;

    float train(const ComplexSampleMatrix& rxSigTraining, const ComplexSampleVector& txSigTraining,
                NomaValSet valSet = std::nullopt) override
    {
        if (numUsers_ != 1) throw std::invalid_argument("multi-user detector: use trainUsers");
        if (!valSet) return trainUsers(rxSigTraining, {txSigTraining});
        NomaTrainHistory& hist = std::get<0>(*valSet);
        size_t P = 0, S = 0;
        std::vector<ComplexSample> rx = detail::flatten(rxSigTraining, numAntennas_, &P);
        std::vector<ComplexSample> rxv = detail::flatten(std::get<1>(*valSet), numAntennas_, &S);
        const ComplexSampleVector& txv = std::get<2>(*valSet);
        if (txSigTraining.size() != P) throw std::invalid_argument("pilot vector length differs from rxSigTraining");
        if (txv.size() != S) throw std::invalid_argument("validation symbols differ in length from their samples");
        if (P == 0) throw std::invalid_argument("no training samples");
        const uint32_t steps = apsm_train_steps(h_, uint32_t(P));
        std::vector<float> out(size_t(steps) * 6 + 6);
        uint32_t n = 0;
        float ms = 0.f;
        detail::throw_status(apsm_train_history(h_, reinterpret_cast<const float*>(rx.data()),
                                                reinterpret_cast<const float*>(txSigTraining.data()), uint32_t(P),
                                                reinterpret_cast<const float*>(rxv.data()),
                                                reinterpret_cast<const float*>(txv.data()), uint32_t(S),
                                                hist.bitPerSymbol, hist.modulationScale, out.data(), steps, &n, &ms),
                             apsm_last_error(h_));
        for (uint32_t t = 0; t < n; ++t) {
            const float* r = &out[size_t(t) * 6];
            hist.evmTrain.push_back(r[0]);
            hist.serTrain.push_back(r[1]);
            hist.berTrain.push_back(r[2]);
            hist.evmVal.push_back(r[3]);
            hist.serVal.push_back(r[4]);
            hist.berVal.push_back(r[5]);
        }
        return ms;
    }

    float detect(const ComplexSampleMatrix& rxSigData, ComplexSampleVector& estData) override
    {
        if (numUsers_ != 1) throw std::invalid_argument("multi-user detector: use detectUsers");
        std::vector<ComplexSampleVector> est;
        float ms = detectUsers(rxSigData, est);
        estData = std::move(est[0]);
        return ms;
    }

    void resetState() override { detail::throw_status(apsm_reset(h_), apsm_last_error(h_)); }

    // tx: one pilot vector per user (all of length P)
    float trainUsers(const ComplexSampleMatrix& rxSigTraining, const std::vector<ComplexSampleVector>& txSigTraining)
    {
        size_t P = 0;
        std::vector<ComplexSample> rx = detail::flatten(rxSigTraining, numAntennas_, &P);
        if (txSigTraining.size() != numUsers_) throw std::invalid_argument("need one pilot vector per user");
        std::vector<ComplexSample> tx;
        tx.reserve(numUsers_ * P);
        for (const auto& t : txSigTraining) {
            if (t.size() != P) throw std::invalid_argument("pilot vector length differs from rxSigTraining");
            tx.insert(tx.end(), t.begin(), t.end());
        }
        if (P == 0) throw std::invalid_argument("no training samples");
        float ms = 0.f;
        detail::throw_status(apsm_train(h_, reinterpret_cast<const float*>(rx.data()),
                                        reinterpret_cast<const float*>(tx.data()), uint32_t(P), &ms),
                             apsm_last_error(h_));
        return ms;
    }

    float detectUsers(const ComplexSampleMatrix& rxSigData, std::vector<ComplexSampleVector>& estData)
    {
        size_t S = 0;
        std::vector<ComplexSample> rx = detail::flatten(rxSigData, numAntennas_, &S);
        std::vector<ComplexSample> est(size_t(numUsers_) * S);
        float ms = 0.f;
        if (S)
            detail::throw_status(apsm_detect(h_, reinterpret_cast<const float*>(rx.data()), uint32_t(S),
                                             reinterpret_cast<float*>(est.data()), &ms),
                                 apsm_last_error(h_));
        estData.assign(numUsers_, ComplexSampleVector());
        for (uint32_t u = 0; u < numUsers_; ++u)
            estData[u].assign(est.begin() + ptrdiff_t(u * S), est.begin() + ptrdiff_t((u + 1) * S));
        return ms;
    }

    apsm_detector* handle() { return h_; }

private:
    apsm_detector* h_ = nullptr;
    uint32_t numAntennas_;
    uint32_t numUsers_;
};

class NomaDetectorFactory {
public:
    static std::unique_ptr<NomaDetector> build(const std::string& algorithmConfig, uint32_t numAntennas)
    {
        return std::unique_ptr<NomaDetector>(new ApsmB200Detector(algorithmConfig, numAntennas));
    }
    template <class Json> static std::unique_ptr<NomaDetector> build(const Json& algorithmConfig, uint32_t numAntennas)
    {
        return build(std::string(algorithmConfig.dump()), numAntennas);
    }
};

} // namespace apsm_b200
