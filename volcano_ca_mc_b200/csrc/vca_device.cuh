// vca_device.cuh -- device primitives shared by the CA and MC kernels (sm_100a).
//
// Hash: the reference's stateless splitmix64 cascade (engine/src/core/Rng.hpp:35-74), restated as
// 64-bit integer code so every random decision is bit-identical to the CPU engine.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace vca {

// CellType (engine/src/core/Types.hpp:13-19).
constexpr uint8_t kAir = 0, kRock = 1, kLava = 2, kBasalt = 3, kVoid = 255;

// Salts (engine/src/core/Rng.hpp:22-31).
constexpr uint64_t kSaltNeighborhood = 0x4E45494748424F52ULL;
constexpr uint64_t kSaltTieBreak = 0x5449455F42524B31ULL;
constexpr uint64_t kSaltMcInit = 0x4D43494E49544F52ULL;
constexpr uint64_t kSaltMcMobility = 0x4D434D4F42494C49ULL;
constexpr uint64_t kSaltMcOrient = 0x4D434F5249454E54ULL;
constexpr uint64_t kSaltMcAccept = 0x4D43414343455054ULL;

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ uint64_t hash_prefix(uint64_t seed, uint64_t step) {
    return splitmix64(splitmix64(seed ^ 0xA0761D6478BD642FULL) ^ step);
}
__host__ __device__ __forceinline__ uint64_t hash_index(uint64_t prefix, uint64_t idx) { return splitmix64(prefix ^ idx); }
__host__ __device__ __forceinline__ uint64_t hash_salt(uint64_t h, uint64_t salt) { return splitmix64(h ^ salt); }

// x mod d for a 64-bit x and a divisor 1 <= d < 2^32, exact: q = floor(x * m / 2^64) with
// m = floor((2^64 - 1) / d) underestimates floor(x / d) by at most 2, so the remainder
// x - q*d lies in [0, 3d) and at most two subtractions finish it.
struct FastMod {
    uint64_t d;
    uint64_t m;
};
inline FastMod make_fastmod(uint64_t d) { return FastMod{d, d ? ~0ULL / d : 0}; }
__device__ __forceinline__ uint64_t fast_mod(uint64_t x, FastMod f) {
    const uint64_t q = __umul64hi(x, f.m);
    uint64_t r = x - q * f.d;
    if (r >= f.d) r -= f.d;
    if (r >= f.d) r -= f.d;
    return r;
}

// n / d and n % d for 32-bit n and a divisor d >= 1 fixed at set-up: q = umulhi(n, m) with
// m = floor((2^32 - 1) / d) is floor(n / d) or one less, one correction step finishes it.
struct FastDiv32 {
    uint32_t d;
    uint32_t m;
};
inline FastDiv32 make_fastdiv32(uint32_t d) { return FastDiv32{d, d ? 0xFFFFFFFFu / d : 0u}; }
__device__ __forceinline__ uint32_t fast_divmod(uint32_t n, FastDiv32 f, uint32_t& rem) {
    uint32_t q = __umulhi(n, f.m);
    uint32_t r = n - q * f.d;
    if (r >= f.d) {
        ++q;
        r -= f.d;
    }
    rem = r;
    return q;
}

// Offsets of the neighbourhood variants (engine/src/core/Neighborhood.cpp:55-119).
struct NbTable {
    int variants;
    int count[6];
    int8_t off[6][26][3];
};

}  // namespace vca
