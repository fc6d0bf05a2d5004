// Shared device/host definitions for the B200 VIA answer path.
//
// Modular arithmetic follows the reference's contract (canonical residues in
// [0, q), crates/via-primitives/src/algebra/zq/modulus.rs:45-211); the internal
// reduction methods (Shoup products for fixed multipliers, lazy 128-bit sums
// reduced once) are this build's own and exact, so every coefficient-form
// output equals the reference's.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>

typedef uint64_t u64;
typedef int64_t i64;
typedef uint32_t u32;
typedef unsigned __int128 u128;
typedef __int128 i128;

namespace via {

struct CudaError : std::runtime_error {
  int status;
  CudaError(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define VIA_CUDA(call)                                                                              \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess)                                                                          \
      throw ::via::CudaError(102, std::string(#call) + ": " + cudaGetErrorString(e_) + " @ " +     \
                                      __FILE__ + ":" + std::to_string(__LINE__));                   \
  } while (0)

// Kernel launches issued by this library (reported by via_kernel_launches()).
extern unsigned long long g_kernel_launches;
#define VIA_LAUNCHED()                               \
  do {                                               \
    __atomic_add_fetch(&::via::g_kernel_launches, 1, __ATOMIC_RELAXED); \
    VIA_CUDA(cudaGetLastError());                    \
  } while (0)

// A modulus with the constants every kernel needs. `q` < 2^63.
struct DevMod {
  u64 q;
  u64 barrett;    // floor((2^64 - 1) / q), 64-bit Barrett for x < 2^64
  u64 r64;        // 2^64 mod q
  u64 r64_shoup;  // floor(r64 * 2^64 / q)
  int log2q;      // >= 0 when q is a power of two
  int pad;
};

inline DevMod make_devmod(u64 q) {
  DevMod m;
  m.q = q;
  m.log2q = ((q & (q - 1)) == 0) ? __builtin_ctzll(q) : -1;
  m.barrett = ~(u64)0 / q;
  m.r64 = (u64)(((u128)1 << 64) % q);
  m.r64_shoup = (u64)(((u128)m.r64 << 64) / q);
  m.pad = 0;
  return m;
}

__host__ __device__ __forceinline__ u64 mulhi(u64 a, u64 b) {
#ifdef __CUDA_ARCH__
  return __umul64hi(a, b);
#else
  return (u64)(((u128)a * b) >> 64);
#endif
}

// x mod q for x < 2^64.
__host__ __device__ __forceinline__ u64 reduce64(u64 x, const DevMod& m) {
  if (m.log2q >= 0) return x & (m.q - 1);
  u64 qe = mulhi(x, m.barrett);
  u64 r = x - qe * m.q;
  if (r >= m.q) r -= m.q;
  if (r >= m.q) r -= m.q;
  return r;
}

// Shoup product a*w mod q with ws = floor(w * 2^64 / q), a < 2^64, w < q.
__host__ __device__ __forceinline__ u64 mul_shoup(u64 a, u64 w, u64 ws, u64 q) {
  u64 t = mulhi(a, ws);
  u64 r = a * w - t * q;
  return r >= q ? r - q : r;
}

// (hi:lo) mod q for any 128-bit value: hi*2^64 + lo with hi reduced first.
__host__ __device__ __forceinline__ u64 reduce128(u64 hi, u64 lo, const DevMod& m) {
  if (m.log2q >= 0) return lo & (m.q - 1);
  u64 h = reduce64(hi, m);
  u64 t = mul_shoup(h, m.r64, m.r64_shoup, m.q);  // h * 2^64 mod q
  u64 l = reduce64(lo, m);
  u64 s = t + l;
  return s >= m.q ? s - m.q : s;
}

__host__ __device__ __forceinline__ u64 mulmod(u64 a, u64 b, const DevMod& m) {
  if (m.log2q >= 0) return (a * b) & (m.q - 1);
  return reduce128(mulhi(a, b), a * b, m);
}

__host__ __device__ __forceinline__ u64 addmod(u64 a, u64 b, u64 q) {
  u64 s = a + b;
  return s >= q ? s - q : s;
}
__host__ __device__ __forceinline__ u64 submod(u64 a, u64 b, u64 q) { return a >= b ? a - b : a + (q - b); }
__host__ __device__ __forceinline__ u64 negmod(u64 a, u64 q) { return a == 0 ? 0 : q - a; }

// 128-bit accumulator.
struct Acc128 {
  u64 lo, hi;
};
__host__ __device__ __forceinline__ void mac128(Acc128& acc, u64 a, u64 b) {
  u64 pl = a * b, ph = mulhi(a, b);
  u64 nl = acc.lo + pl;
  acc.hi += ph + (nl < pl ? 1 : 0);
  acc.lo = nl;
}

// Signed residue lift of a small integer into [0, q).
__host__ __device__ __forceinline__ u64 lift_i64(i64 v, const DevMod& m) {
  if (v >= 0) return (u64)v < m.q ? (u64)v : reduce64((u64)v, m);
  const u64 a = (u64)(-v);
  if (a < m.q) return m.q - a;  // a > 0
  u64 r = reduce64(a, m);
  return r == 0 ? 0 : m.q - r;
}

}  // namespace via
