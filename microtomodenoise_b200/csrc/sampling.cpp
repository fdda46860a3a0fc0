#include "sampling.hpp"

#include <algorithm>
#include <cmath>

namespace inlm {

GlibcRand::GlibcRand(unsigned int seed) {
    if (seed == 0) seed = 1;
    int32_t r[34];
    r[0] = (int32_t)seed;
    int32_t word = (int32_t)seed;
    for (int i = 1; i < 31; i++) {
        int64_t hi = word / 127773;
        int64_t lo = word % 127773;
        word = (int32_t)(16807 * lo - 2836 * hi);
        if (word < 0) word += 2147483647;
        r[i] = word;
    }
    for (int i = 31; i < 34; i++) r[i] = r[i - 31];
    for (int i = 0; i < 34; i++) r_[i] = (uint32_t)r[i];
    head_ = 0;
    for (int i = 0; i < 310; i++) next();
}

int GlibcRand::next() {
    // ring holds r[i-34..i-1] starting at head_
    uint32_t v = r_[(head_ + 31) % 34] + r_[(head_ + 3) % 34];
    r_[head_] = v;  // overwrite r[i-34]
    head_ = (head_ + 1) % 34;
    return (int)(v >> 1);
}

std::vector<long long> draw_noise_samples(const int shape[3], uint64_t n_samples, int patchsize,
                                          int circular_mask_diameter, unsigned int seed) {
    const int nx = shape[0], ny = shape[1], nz = shape[2];
    const long long nslice = (long long)nx * ny;
    // float maxradiussq = d/2.f - sqrt(2*ps*ps) (double), squared in float
    float maxradiussq =
        (float)((double)(circular_mask_diameter / 2.f) - std::sqrt((double)(2 * patchsize * patchsize)));
    maxradiussq *= maxradiussq;
    GlibcRand rng(seed);
    std::vector<long long> out(n_samples);
    for (uint64_t s = 0; s < n_samples; s++) {
        int x = rng.next() % (nx - patchsize);
        int y = rng.next() % (ny - patchsize);
        int z = rng.next() % nz;
        if (circular_mask_diameter > 0) {
            float rsq = (float)((x - nx / 2) * (x - nx / 2) + (y - ny / 2) * (y - ny / 2));
            while (rsq > maxradiussq) {
                x = rng.next() % (nx - patchsize);
                y = rng.next() % (ny - patchsize);
                rsq = (float)((x - nx / 2) * (x - nx / 2) + (y - ny / 2) * (y - ny / 2));
            }
        }
        out[s] = z * nslice + (long long)y * nx + x;
    }
    std::sort(out.begin(), out.end());
    return out;
}

void noise_zwindows(const std::vector<long long>& samples, const int shape[3], int windowsize,
                    std::vector<int>& start, std::vector<int>& end) {
    const long long nslice = (long long)shape[0] * shape[1];
    const long long n = (long long)samples.size();
    start.assign(shape[2], 0);
    end.assign(shape[2], 0);
    int sp = 0, ep = 0;
    for (int pos = 0; pos < shape[2]; pos++) {
        while (sp < n - 1 && samples[sp] / nslice <= (pos - windowsize / 2)) sp++;
        while (ep < (int)(n - 1) && samples[ep] / nslice <= (pos + windowsize / 2)) ep++;
        start[pos] = sp;
        end[pos] = ep;
    }
}

}  // namespace inlm
