// Drives the C++ drop-in header (include/apsm_b200.hpp) the way the
// reference CLI drives its NomaDetector (cpp/cli/detect/noma_detect.cpp:
// 130-137): build from an algorithm JSON, train on pilots, detect data.
// Usage: cpp_api_check <json> <N> <P> <S> <rx_train.f32> <tx.f32> <rx_data.f32> <est_out.f32>
//                      [<tx_data.f32> <history.csv>]
// With the last two arguments training takes the data as its validation set
// (NomaValSet, as the CLI's -th option) and the history is written as CSV.
// The float files hold interleaved complex64 samples (antenna-major for rx).
#include "apsm_b200.hpp"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>

using namespace apsm_b200;

static std::vector<ComplexSample> read_c64(const char* path, size_t n)
{
    std::vector<ComplexSample> v(n);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char*>(v.data()), std::streamsize(n * sizeof(ComplexSample)));
    if (!f) throw std::runtime_error(std::string("cannot read ") + path);
    return v;
}

int main(int argc, char** argv)
{
    if (argc == 2) {
        // configuration check only: prints the factory's exception message
        try {
            NomaDetectorFactory::build(std::string(argv[1]), 8);
            std::cout << "ok" << std::endl;
            return 0;
        } catch (const std::invalid_argument& e) {
            std::cout << "invalid_argument: " << e.what() << std::endl;
            return 3;
        } catch (const std::exception& e) {
            std::cout << "error: " << e.what() << std::endl;
            return 4;
        }
    }
    if (argc != 9 && argc != 11) {
        std::cerr << "usage: cpp_api_check json N P S rx_train tx rx_data est_out [tx_data history.csv]" << std::endl;
        return 2;
    }
    const uint32_t N = uint32_t(std::atoi(argv[2])), P = uint32_t(std::atoi(argv[3])), S = uint32_t(std::atoi(argv[4]));
    auto rxt = read_c64(argv[5], size_t(N) * P);
    auto tx = read_c64(argv[6], P);
    auto rxd = read_c64(argv[7], size_t(N) * S);
    ComplexSampleMatrix rxTraining(N), rxData(N);
    for (uint32_t a = 0; a < N; ++a) {
        rxTraining[a].assign(rxt.begin() + ptrdiff_t(a) * P, rxt.begin() + ptrdiff_t(a + 1) * P);
        rxData[a].assign(rxd.begin() + ptrdiff_t(a) * S, rxd.begin() + ptrdiff_t(a + 1) * S);
    }
    std::unique_ptr<NomaDetector> d = NomaDetectorFactory::build(std::string(argv[1]), N);
    NomaTrainHistory stats(2, 0.70710677f); // QPSK
    NomaValSet valSet = std::nullopt;
    ComplexSampleVector txData;
    if (argc == 11) {
        txData = read_c64(argv[9], S);
        valSet.emplace(std::make_tuple(std::ref(stats), std::cref(rxData), std::cref(txData)));
    }
    float trainTime = d->train(rxTraining, tx, valSet);
    if (valSet.has_value()) std::get<0>(*valSet).toCsv(argv[10]);
    ComplexSampleVector est;
    float detectTime = d->detect(rxData, est);
    std::cout << "Train time = " << trainTime << " ms, detect time = " << detectTime << " ms" << std::endl;
    std::ofstream o(argv[8], std::ios::binary);
    o.write(reinterpret_cast<const char*>(est.data()), std::streamsize(est.size() * sizeof(ComplexSample)));
    return 0;
}
