// Random streams for the CPU oracle (test infrastructure only).
//
// Two streams are restated here:
//
//  1. The reference's stream.  coretrace/mtrand.h:136-139,298-343 wraps
//     std::default_random_engine (libstdc++: minstd_rand0, x <- 16807 x mod 2^31-1),
//     std::uniform_real_distribution<double>(0,1) and std::normal_distribution<double>(0,1).
//     libstdc++ (GCC 13) builds a uniform double from two engine outputs
//     (generate_canonical<double,53>: (u0-1) + (u1-1)*R, divided by R^2, R = 2^31-2,
//     clamped below 1), and draws normals with the Marsaglia polar method, returning
//     y*mult and caching x*mult for the next call.  Replaying this stream lets the
//     restatement reproduce a reference run record for record.
//
//  2. The per-ray counter-based stream used by the CUDA product: Philox4x32-10
//     (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
//     SC'11).  Draw k of ray s is taken from block k/2 of the counter
//     {k/2, s_lo, s_hi, 0x5B200} under key {seed, 0x50C7A5E1}.  Even k uses output
//     words 0,1 and odd k words 2,3; a double in [0,1) takes 27 bits of the first word
//     and 26 of the second (53 bits), times 2^-53.
#pragma once
#include <cstdint>
#include <cmath>

namespace st_oracle_rng {

// ---- libstdc++ minstd_rand0 + generate_canonical + polar normal -------------------
struct Minstd {
    uint64_t x = 1;
    bool saved_ok = false;
    double saved = 0.0;

    void seed(uint64_t s) {
        x = s % 2147483647ULL;
        if (x == 0) x = 1;
        saved_ok = false;
    }
    uint64_t next() {
        x = (x * 16807ULL) % 2147483647ULL;
        return x;
    }
    double uniform() {
        const double r = 2147483646.0;  // max - min + 1 of minstd (min = 1)
        double sum = 0.0, mult = 1.0;
        for (int k = 0; k < 2; ++k) {
            sum += double(next() - 1) * mult;
            mult *= r;
        }
        double ret = sum / mult;
        if (ret >= 1.0) ret = std::nextafter(1.0, 0.0);
        return ret;
    }
    // N(0,1) by the polar method with one cached value.
    double normal() {
        if (saved_ok) {
            saved_ok = false;
            return saved;
        }
        double x1, y1, r2;
        do {
            x1 = 2.0 * uniform() - 1.0;
            y1 = 2.0 * uniform() - 1.0;
            r2 = x1 * x1 + y1 * y1;
        } while (r2 > 1.0 || r2 == 0.0);
        const double mult = std::sqrt(-2.0 * std::log(r2) / r2);
        saved = x1 * mult;
        saved_ok = true;
        return y1 * mult;
    }
};

// ---- Philox4x32-10 ------------------------------------------------------------------
inline void philox4x32_10(uint32_t ctr[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = uint64_t(M0) * ctr[0];
        const uint64_t p1 = uint64_t(M1) * ctr[2];
        const uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
        const uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
        const uint32_t n0 = hi1 ^ ctr[1] ^ k0;
        const uint32_t n2 = hi0 ^ ctr[3] ^ k1;
        ctr[0] = n0;
        ctr[1] = lo1;
        ctr[2] = n2;
        ctr[3] = lo0;
        k0 += W0;
        k1 += W1;
    }
}

constexpr uint32_t kPhiloxKey1 = 0x50C7A5E1u;
constexpr uint32_t kPhiloxTag = 0x0005B200u;

// Two 32-bit words -> double in [0,1) with 53 random bits.
inline double words_to_unit(uint32_t a, uint32_t b) {
    const uint64_t m = (uint64_t(a >> 5) << 26) | uint64_t(b >> 6);
    return double(m) * (1.0 / 9007199254740992.0);
}

// Draw number k (0-based) of the stream that belongs to ray s under 'seed'.
inline double philox_draw(uint32_t seed, uint64_t s, uint32_t k) {
    uint32_t c[4] = {k >> 1, uint32_t(s), uint32_t(s >> 32), kPhiloxTag};
    philox4x32_10(c, seed, kPhiloxKey1);
    return (k & 1u) ? words_to_unit(c[2], c[3]) : words_to_unit(c[0], c[1]);
}

}  // namespace st_oracle_rng
