// Noise-sample positions (Noise/noiselevel.cpp:192-234) drawn on the host
// with a generator that reproduces glibc's rand() sequence, so a seed gives
// the positions the reference draws after srand(seed) with one thread.
#pragma once

#include <cstdint>
#include <vector>

namespace inlm {

// glibc random_r TYPE_3 (additive feedback, degree 31, separation 3):
// r[0] = seed (1 if 0), r[i] = 16807 r[i-1] mod (2^31-1) (Schrage) for
// i < 31, r[31..33] = r[0..2], r[i] = r[i-3] + r[i-31] mod 2^32 afterwards;
// the k-th output is r[k+344] >> 1 (the first 310 are discarded).
class GlibcRand {
  public:
    explicit GlibcRand(unsigned int seed);
    int next();

  private:
    uint32_t r_[34];
    int head_ = 0;  // ring position of r[i-34]
};

// drawsamples with the sequential rand() order, sorted ascending.
std::vector<long long> draw_noise_samples(const int shape[3], uint64_t n_samples, int patchsize,
                                          int circular_mask_diameter, unsigned int seed);

// z windows (noiselevel.cpp:538-546): for every slice the inclusive sample
// range [start, end]; end stops on the first sample past the window, which
// the reference includes.
void noise_zwindows(const std::vector<long long>& samples, const int shape[3], int windowsize,
                    std::vector<int>& start, std::vector<int>& end);

}  // namespace inlm
