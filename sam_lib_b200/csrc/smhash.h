// Content hash of an SM array (NEQ + NZEROL doubles), the same on the host and
// on the device: H = sum over i of mix(word_i, i) modulo 2^64, with mix the
// splitmix64 finaliser of the word and its position.  The sum is order-free,
// so any parallel reduction (GPU atomics, host threads) gives the same value,
// and an edit of any entry changes H except with probability 2^-64.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define SMHASH_HD __host__ __device__ __forceinline__
#else
#define SMHASH_HD inline
#endif

namespace sprb {

SMHASH_HD uint64_t sm_mix(uint64_t w, uint64_t i) {
    uint64_t z = w ^ (i * 0x9e3779b97f4a7c15ULL + 0x632be59bd9b4e019ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// Host: the hash of n doubles with up to `threads` threads.
uint64_t sm_hash_host(const double* a, int64_t n, int threads);

}  // namespace sprb
