// The reference's PRG (crates/via-primitives/src/sampling/prg.rs:57-205, SHAKE-256
// from the sha3 0.10.9 / keccak 0.1.6 crates): counter mode,
// block b = SHAKE256(seed || le64(b))[0..136), bytes served in order. Keccak-f[1600]
// is written from FIPS 202. Shared by the wire decoder and the device client.
#pragma once
#include <stdint.h>

#include "common.cuh"

namespace via {

constexpr int SHAKE_RATE = 136;  // bytes per block (SHAKE256)
constexpr int RATE_LANES = SHAKE_RATE / 8;

// Keccak-f[1600] (FIPS 202 section 3): round constants from the rc(t) LFSR
// (Algorithm 5) and rotation offsets from the (x, y) -> (y, 2x + 3y) walk
// (Algorithm 2), both evaluated at compile time.
struct KeccakConsts {
  u64 rc[24];
  int rot[25];
};

constexpr bool rc_bit(int t) {
  if (t % 255 == 0) return true;
  unsigned r = 1;  // R = 10000000 as bits r0..r7 with r0 the low bit
  for (int i = 1; i <= t % 255; ++i) {
    // R = 0 || R, then r0 ^= r8, r4 ^= r8, r5 ^= r8, r6 ^= r8, R = Trunc8(R).
    r <<= 1;
    const unsigned r8 = (r >> 8) & 1;
    r ^= r8;
    r ^= r8 << 4;
    r ^= r8 << 5;
    r ^= r8 << 6;
    r &= 0xFF;
  }
  return r & 1;
}

constexpr KeccakConsts make_keccak_consts() {
  KeccakConsts k{};
  for (int i = 0; i < 24; ++i) {
    u64 c = 0;
    for (int j = 0; j <= 6; ++j)
      if (rc_bit(j + 7 * i)) c |= (u64)1 << ((1 << j) - 1);
    k.rc[i] = c;
  }
  for (int i = 0; i < 25; ++i) k.rot[i] = 0;
  int x = 1, y = 0;
  for (int t = 0; t < 24; ++t) {
    k.rot[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
    const int nx = y, ny = (2 * x + 3 * y) % 5;
    x = nx;
    y = ny;
  }
  return k;
}

static __constant__ KeccakConsts c_keccak = make_keccak_consts();

__host__ __device__ inline const KeccakConsts& keccak_consts() {
#ifdef __CUDA_ARCH__
  return c_keccak;
#else
  static constexpr KeccakConsts k = make_keccak_consts();
  return k;
#endif
}

__host__ __device__ __forceinline__ u64 rotl64(u64 v, int s) { return s == 0 ? v : (v << s) | (v >> (64 - s)); }

__host__ __device__ inline void keccak_f1600(u64 (&A)[25]) {
  const KeccakConsts& K = keccak_consts();
  for (int r = 0; r < 24; ++r) {
    u64 C[5], D[5], B[25];
#pragma unroll
    for (int x = 0; x < 5; ++x) C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
#pragma unroll
    for (int x = 0; x < 5; ++x) D[x] = C[(x + 4) % 5] ^ rotl64(C[(x + 1) % 5], 1);
#pragma unroll
    for (int i = 0; i < 25; ++i) A[i] ^= D[i % 5];
#pragma unroll
    for (int x = 0; x < 5; ++x)
#pragma unroll
      for (int y = 0; y < 5; ++y) B[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(A[x + 5 * y], K.rot[x + 5 * y]);
#pragma unroll
    for (int x = 0; x < 5; ++x)
#pragma unroll
      for (int y = 0; y < 5; ++y) A[x + 5 * y] = B[x + 5 * y] ^ (~B[(x + 1) % 5 + 5 * y] & B[(x + 2) % 5 + 5 * y]);
    A[0] ^= K.rc[r];
  }
}

// One PRG block: SHAKE256(seed || le64(counter)) truncated to 136 bytes, as 17
// little-endian lanes. seed || counter (at most 72 bytes) fits one absorbed block.
__host__ __device__ inline void prg_block(const uint8_t* seed, int seed_len, u64 counter, u64 (&out)[RATE_LANES]) {
  u64 A[25];
#pragma unroll
  for (int i = 0; i < 25; ++i) A[i] = 0;
  uint8_t msg[SHAKE_RATE];
  for (int i = 0; i < SHAKE_RATE; ++i) msg[i] = 0;
  for (int i = 0; i < seed_len; ++i) msg[i] = seed[i];
  for (int i = 0; i < 8; ++i) msg[seed_len + i] = (uint8_t)(counter >> (8 * i));
  msg[seed_len + 8] ^= 0x1F;        // SHAKE domain bits and the first pad bit
  msg[SHAKE_RATE - 1] ^= 0x80;      // last pad bit
  for (int l = 0; l < RATE_LANES; ++l) {
    u64 v = 0;
    for (int b = 0; b < 8; ++b) v |= (u64)msg[8 * l + b] << (8 * b);
    A[l] ^= v;
  }
  keccak_f1600(A);
#pragma unroll
  for (int l = 0; l < RATE_LANES; ++l) out[l] = A[l];
}

}  // namespace via
