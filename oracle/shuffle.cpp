// TEST INFRASTRUCTURE ONLY.
// NomaDetector::shuffleData (cpp/lib/noma/noma_detector.cu:59-74): an mt19937
// seeded with seed_seq{1..8}; rx rows and tx are shuffled with copies of the
// same engine, i.e. by one permutation.  perm[i] = original index of sample i.
#include <algorithm>
#include <cstdint>
#include <random>
#include <vector>

extern "C" void apsm_oracle_shuffle_permutation(uint32_t P, int32_t* perm)
{
    std::seed_seq seed{1, 2, 3, 4, 5, 6, 7, 8};
    std::mt19937 base(seed);
    std::vector<int32_t> v(P);
    for (uint32_t i = 0; i < P; ++i) v[i] = int32_t(i);
    std::mt19937 rng = base;
    std::shuffle(v.begin(), v.end(), rng);
    std::copy(v.begin(), v.end(), perm);
}
