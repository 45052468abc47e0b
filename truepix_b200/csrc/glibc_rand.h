// glibc rand() as an explicit generator state (host code).
#pragma once
#include <stdint.h>

namespace tp {

// glibc rand(): the TYPE_3 additive generator (degree 31, separation 3) that
// glibc uses by default. Seeded like srand(seed): r[0] = seed, r[i] = 16807 *
// r[i-1] mod (2^31 - 1) for i < 31, r[31..33] = r[0..2], then 310 outputs are
// discarded; each output is o[i] = o[i-31] + o[i-3] (mod 2^32), returned >> 1.
// The reference never seeds it, so its stream is that of seed 1.
class GlibcRand {
public:
    explicit GlibcRand(uint32_t seed)
    {
        int64_t v = seed;
        s_[0] = (uint32_t)v;
        for (int i = 1; i < 31; ++i) {
            v = (16807 * v) % 2147483647;
            if (v < 0) v += 2147483647;
            s_[i] = (uint32_t)v;
        }
        for (int i = 31; i < 34; ++i) s_[i] = s_[i - 31];
        pos_ = 34;
        for (int i = 0; i < 310; ++i) step();
    }
    int next() { return (int)(step() >> 1); }

private:
    uint32_t step()
    {
        const uint32_t o = s_[(pos_ - 31) % 34] + s_[(pos_ - 3) % 34];
        s_[pos_ % 34] = o;
        ++pos_;
        return o;
    }
    uint32_t s_[34];
    long long pos_;
};

}  // namespace tp
