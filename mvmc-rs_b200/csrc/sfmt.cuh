// SFMT19937 for host and device: C-exact gen_rand32 / genrand_real2 of the SFMT
// library used by mVMC (MEXP 19937, POS1 122, SL1 18, SL2 1 byte, SR1 11, SR2 1 byte,
// little-endian 128-bit lanes; crates/sfmt19937/src/{state,init,real}.rs of
// AtelierArith/mvmc-rs). The 624-word state of a walker lives in shared memory while the
// walker is resident; gen_all refreshes the block of 624 words in one serial pass.
#pragma once

#include <stdint.h>

namespace mvmcb {

constexpr int kSfmtN32 = 624;

__host__ __device__ inline void sfmt_recursion(uint32_t* r, const uint32_t* a, const uint32_t* b,
                                               const uint32_t* c, const uint32_t* d) {
  const uint64_t ah = (static_cast<uint64_t>(a[3]) << 32) | a[2];
  const uint64_t al = (static_cast<uint64_t>(a[1]) << 32) | a[0];
  const uint64_t xh = (ah << 8) | (al >> 56), xl = al << 8;
  const uint64_t ch = (static_cast<uint64_t>(c[3]) << 32) | c[2];
  const uint64_t cl = (static_cast<uint64_t>(c[1]) << 32) | c[0];
  const uint64_t yh = ch >> 8, yl = (cl >> 8) | (ch << 56);
  r[0] = a[0] ^ static_cast<uint32_t>(xl) ^ ((b[0] >> 11) & 0xdfffffefu) ^ static_cast<uint32_t>(yl) ^ (d[0] << 18);
  r[1] = a[1] ^ static_cast<uint32_t>(xl >> 32) ^ ((b[1] >> 11) & 0xddfecb7fu) ^ static_cast<uint32_t>(yl >> 32) ^ (d[1] << 18);
  r[2] = a[2] ^ static_cast<uint32_t>(xh) ^ ((b[2] >> 11) & 0xbffaffffu) ^ static_cast<uint32_t>(yh) ^ (d[2] << 18);
  r[3] = a[3] ^ static_cast<uint32_t>(xh >> 32) ^ ((b[3] >> 11) & 0xbffffff6u) ^ static_cast<uint32_t>(yh >> 32) ^ (d[3] << 18);
}

// Regenerate all 624 words in place (gen_rand_all).
__host__ __device__ inline void sfmt_gen_all(uint32_t* s) {
  constexpr int N = 156, POS1 = 122;
  const uint32_t* r1 = s + 4 * (N - 2);
  const uint32_t* r2 = s + 4 * (N - 1);
  for (int i = 0; i < N; ++i) {
    const int bi = i < N - POS1 ? i + POS1 : i + POS1 - N;
    uint32_t out[4];
    sfmt_recursion(out, s + 4 * i, s + 4 * bi, r1, r2);
    s[4 * i + 0] = out[0];
    s[4 * i + 1] = out[1];
    s[4 * i + 2] = out[2];
    s[4 * i + 3] = out[3];
    r1 = r2;
    r2 = s + 4 * i;
  }
}

__host__ __device__ inline void sfmt_seed(uint32_t* s, int* idx, uint32_t seed) {
  s[0] = seed;
  for (int i = 1; i < kSfmtN32; ++i) s[i] = 1812433253u * (s[i - 1] ^ (s[i - 1] >> 30)) + static_cast<uint32_t>(i);
  *idx = kSfmtN32;
  const uint32_t parity[4] = {0x00000001u, 0x00000000u, 0x00000000u, 0x13c9e684u};
  uint32_t inner = 0;
  for (int i = 0; i < 4; ++i) inner ^= s[i] & parity[i];
  for (int i = 16; i > 0; i >>= 1) inner ^= inner >> i;
  if (inner & 1u) return;
  for (int i = 0; i < 4; ++i) {
    uint32_t work = 1;
    for (int j = 0; j < 32; ++j) {
      if (work & parity[i]) {
        s[i] ^= work;
        return;
      }
      work <<= 1;
    }
  }
}

// One walker's generator: state pointer (shared or host memory), cursor, word count.
struct SfmtRef {
  uint32_t* s;
  int* idx;
  unsigned long long* draws;
  __host__ __device__ uint32_t u32() {
    if (*idx >= kSfmtN32) {
      sfmt_gen_all(s);
      *idx = 0;
    }
    ++*draws;
    return s[(*idx)++];
  }
  __host__ __device__ double real2() { return static_cast<double>(u32()) * (1.0 / 4294967296.0); }
  __host__ __device__ uint32_t mod(uint32_t n) { return u32() % n; }
};

}  // namespace mvmcb
