// oracle/rng_oracle.h -- TEST INFRASTRUCTURE (the checker), never linked into the product.
//
// Scalar restatements of the two uniform generators the photon march can consume:
//
//  * SFMT-19937 (M. Saito, M. Matsumoto, "SIMD-oriented Fast Mersenne Twister", MCQMC 2006),
//    with the 64-bit seeding, 64-bit output and float conversion of the reference's SSE build:
//      seeding        renderer/src/rng_sse.cpp:302-311 (init_gen_rand) and :408-410 (seed)
//      period check   renderer/src/rng_sse.cpp:243-266
//      block refresh  renderer/src/rng_sse.cpp:272-289 (gen_rand_all) with the recursion :140-155
//      64-bit draw    renderer/src/rng_sse.cpp:204-212 (gen_rand64), :412-414 (nextULong)
//      float          renderer/include/rng_sse.h:42-49  ((low 32 bits >> 9) | 0x3f800000) - 1
//    The reference reseeds the engine with the photon index for every photon
//    (renderer/src/photon.cpp:313).
//
//  * Philox-4x32-10 (J. Salmon et al., "Parallel random numbers: as easy as 1, 2, 3", SC'11),
//    keyed by (seed, photon index), counter = draw block; 24-bit float conversion.
#pragma once
#include <cstdint>
#include <cstring>

namespace orc {

class Sfmt19937 {
public:
    static constexpr int kWords128 = 156;            // MEXP/128 + 1
    static constexpr int kWords32 = kWords128 * 4;   // 624
    static constexpr int kWords64 = kWords128 * 2;   // 312
    static constexpr int kPos1 = 122, kSl1 = 18, kSr1 = 11;   // SL2 = SR2 = 1 byte
    static constexpr uint32_t kMask[4] = {0xdfffffefu, 0xddfecb7fu, 0xbffaffffu, 0xbffffff6u};
    static constexpr uint32_t kParity[4] = {0x00000001u, 0x00000000u, 0x00000000u, 0x13c9e684u};

    void seed(uint64_t s) {
        uint64_t x = s;
        set64(0, x);
        for (int i = 1; i < kWords64; ++i) {
            x = 6364136223846793005ULL * (x ^ (x >> 62)) + static_cast<uint64_t>(i);
            set64(i, x);
        }
        idx_ = kWords32;
        certify_period();
    }

    uint64_t next_u64() {
        if (idx_ >= kWords32) {
            refresh();
            idx_ = 0;
        }
        uint64_t r = get64(idx_ / 2);
        idx_ += 2;
        return r;
    }

    // The reference's float draw: 23 random mantissa bits, value in [0, 1).
    float next_float() {
        uint32_t bits = (static_cast<uint32_t>(next_u64() & 0xffffffffULL) >> 9) | 0x3f800000u;
        float f;
        std::memcpy(&f, &bits, 4);
        return f - 1.0f;
    }

private:
    uint32_t w_[kWords32];
    int idx_ = -1;

    void set64(int i, uint64_t v) {
        w_[2 * i] = static_cast<uint32_t>(v);
        w_[2 * i + 1] = static_cast<uint32_t>(v >> 32);
    }
    uint64_t get64(int i) const {
        return static_cast<uint64_t>(w_[2 * i]) | (static_cast<uint64_t>(w_[2 * i + 1]) << 32);
    }

    void certify_period() {
        uint32_t inner = 0;
        for (int i = 0; i < 4; ++i) inner ^= w_[i] & kParity[i];
        for (int s = 16; s > 0; s >>= 1) inner ^= inner >> s;
        if (inner & 1u) return;
        for (int i = 0; i < 4; ++i) {
            for (int b = 0; b < 32; ++b) {
                uint32_t bit = 1u << b;
                if (bit & kParity[i]) { w_[i] ^= bit; return; }
            }
        }
    }

    // One 128-bit recursion step: a,b,c,d are 4-lane little-endian 128-bit words.
    static void recursion(const uint32_t *a, const uint32_t *b, const uint32_t *c,
                          const uint32_t *d, uint32_t *out) {
        // c shifted right by 8 bits as a 128-bit integer; a shifted left by 8 bits likewise
        uint32_t cr[4] = {(c[0] >> 8) | (c[1] << 24), (c[1] >> 8) | (c[2] << 24),
                          (c[2] >> 8) | (c[3] << 24), c[3] >> 8};
        uint32_t al[4] = {a[0] << 8, (a[1] << 8) | (a[0] >> 24),
                          (a[2] << 8) | (a[1] >> 24), (a[3] << 8) | (a[2] >> 24)};
        for (int k = 0; k < 4; ++k)
            out[k] = a[k] ^ al[k] ^ cr[k] ^ ((b[k] >> kSr1) & kMask[k]) ^ (d[k] << kSl1);
    }

    void refresh() {
        uint32_t r1[4], r2[4], r[4];
        std::memcpy(r1, &w_[4 * (kWords128 - 2)], 16);
        std::memcpy(r2, &w_[4 * (kWords128 - 1)], 16);
        for (int i = 0; i < kWords128; ++i) {
            int j = i + kPos1;
            if (j >= kWords128) j -= kWords128;   // already refreshed words for the tail
            recursion(&w_[4 * i], &w_[4 * j], r1, r2, r);
            std::memcpy(&w_[4 * i], r, 16);
            std::memcpy(r1, r2, 16);
            std::memcpy(r2, r, 16);
        }
    }
};

struct Philox4x32 {
    static void block(uint32_t ctr[4], uint32_t key0, uint32_t key1) {
        const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
        const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
        uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
        uint32_t k0 = key0, k1 = key1;
        for (int r = 0; r < 10; ++r) {
            uint64_t p0 = static_cast<uint64_t>(M0) * c0;
            uint64_t p1 = static_cast<uint64_t>(M1) * c2;
            uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
            uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
            c0 = hi1 ^ c1 ^ k0;
            c1 = lo1;
            c2 = hi0 ^ c3 ^ k1;
            c3 = lo0;
            k0 += W0;
            k1 += W1;
        }
        ctr[0] = c0; ctr[1] = c1; ctr[2] = c2; ctr[3] = c3;
    }
};

// Per-photon Philox stream: counter (block, 0, photon lo, photon hi), key (seed lo, seed hi).
class PhiloxStream {
public:
    void seed(uint64_t seed, uint64_t photon) {
        key0_ = static_cast<uint32_t>(seed);
        key1_ = static_cast<uint32_t>(seed >> 32);
        ph0_ = static_cast<uint32_t>(photon);
        ph1_ = static_cast<uint32_t>(photon >> 32);
        blk_ = 0;
        have_ = 0;
    }
    float next_float() {
        if (have_ == 0) {
            buf_[0] = blk_++; buf_[1] = 0; buf_[2] = ph0_; buf_[3] = ph1_;
            Philox4x32::block(buf_, key0_, key1_);
            have_ = 4;
        }
        uint32_t x = buf_[4 - have_];
        --have_;
        return static_cast<float>(x >> 8) * (1.0f / 16777216.0f);
    }

private:
    uint32_t key0_ = 0, key1_ = 0, ph0_ = 0, ph1_ = 0, blk_ = 0;
    uint32_t buf_[4] = {0, 0, 0, 0};
    int have_ = 0;
};

}  // namespace orc
