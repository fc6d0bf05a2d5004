// Exact wide arithmetic for the gadget decomposition and modulus switches:
// 128-bit CRT values, round(|c| * B^L / Q) with a 256-bit-equivalent exact
// division, and balanced base-B digits (crates/via-primitives/src/encryption/
// gadget.rs:115-190, crates/via-primitives/src/algebra/wide.rs:145-153).
// Host-callable so the same code is checked against the oracle on the CPU.
#pragma once
#include <cmath>

#include "ntt.cuh"
#include "server.cuh"

namespace via {

// ---------------------------------------------------------------------------
// Exact wide arithmetic helpers (device).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ double u128_to_double(u128 x) {
  return (double)(u64)(x >> 64) * 18446744073709551616.0 + (double)(u64)x;
}
__host__ __device__ __forceinline__ double i128_to_double(i128 x) {
  return x < 0 ? -u128_to_double((u128)(-x)) : u128_to_double((u128)x);
}
__host__ __device__ __forceinline__ u128 double_to_u128(double d) {
  if (d <= 0.0) return 0;
  if (d < 18446744073709551616.0) return (u128)(u64)d;
  double hi = floor(d / 18446744073709551616.0);
  double lo = d - hi * 18446744073709551616.0;
  if (lo < 0) lo = 0;
  return ((u128)(u64)hi << 64) | (u128)(u64)lo;
}

// floor(x / D) for x < 2^127, 0 < D < 2^127, given dD = (double)D. Exact:
// a double estimate, a second estimate from the (small, exact) remainder, then
// a final +-1 fix.
__host__ __device__ __forceinline__ u128 div_exact(u128 x, u128 D, double dD) {
  u128 q = double_to_u128(u128_to_double(x) / dD);
  i128 r = (i128)(x - q * D);
  i128 qci = (i128)(i64)floor(i128_to_double(r) / dD);
  r -= qci * (i128)D;
  q = (u128)((i128)q + qci);
  // The two estimates leave |error| <= 1; the loops are bounded regardless.
  for (int it = 0; it < 4 && r < 0; ++it) {
    r += (i128)D;
    q -= 1;
  }
  for (int it = 0; it < 4 && r >= (i128)D; ++it) {
    r -= (i128)D;
    q += 1;
  }
  return q;
}

// CRT reconstruction (prim/algebra/rns/basis.rs reconstruct).
__host__ __device__ __forceinline__ u128 crt2(u64 a0, u64 a1, const DevRing& R) {
  const DevMod& m1 = R.m[1];
  u64 a0m = reduce64(a0, m1);
  u64 diff = submod(a1, a0m, m1.q);
  u64 t = mul_shoup(diff, R.q0inv_mod_q1, R.q0inv_shoup, m1.q);
  return (u128)a0 + (u128)R.m[0].q * t;
}

// ---------------------------------------------------------------------------
// Division by an invariant 64-bit divisor (Moller and Granlund, "Improved
// division by invariant integers", IEEE Trans. Computers 60(2), 2011,
// Algorithm 4): the divisor is normalized (top bit set) and its reciprocal
// v = floor((2^128 - 1) / d) - 2^64 precomputed, so a 128-by-64 division is two
// multiplications and two fix-ups.
// ---------------------------------------------------------------------------
struct Div64 {
  u64 d = 1;   // divisor
  u64 dn = 0;  // d << s
  u64 v = 0;   // reciprocal of dn
  int s = 0;   // leading zeros of d
};

inline Div64 make_div64(u64 d) {
  Div64 r;
  r.d = d;
  r.s = __builtin_clzll(d);
  r.dn = d << r.s;
  r.v = (u64)((~(u128)0) / r.dn - ((u128)1 << 64));
  return r;
}

// (u1 * 2^64 + u0) / dn for u1 < dn: quotient, remainder in r.
__host__ __device__ __forceinline__ u64 div_2by1(u64 u1, u64 u0, const Div64& D, u64& r) {
  u64 q0 = D.v * u1;
  u64 q1 = mulhi(D.v, u1);
  const u64 s0 = q0 + u0;
  q1 += u1 + (s0 < q0 ? 1 : 0);
  q0 = s0;
  q1 += 1;
  u64 rr = u0 - q1 * D.dn;
  if (rr > q0) {
    q1 -= 1;
    rr += D.dn;
  }
  if (rr >= D.dn) {
    q1 += 1;
    rr -= D.dn;
  }
  r = rr;
  return q1;
}

// floor(n / d) and n mod d for a 128-bit n and a 64-bit divisor.
__host__ __device__ __forceinline__ u128 div128by64(u128 n, const Div64& D, u64& rem) {
  const u64 hi = (u64)(n >> 64), lo = (u64)n;
  const int s = D.s;
  const u64 n2 = s ? hi >> (64 - s) : 0;
  const u64 n1 = s ? (hi << s) | (lo >> (64 - s)) : hi;
  const u64 n0 = lo << s;
  u64 r1, r0;
  const u64 qh = div_2by1(n2, n1, D, r1);
  const u64 ql = div_2by1(r1, n0, D, r0);
  rem = r0 >> s;
  return ((u128)qh << 64) | ql;
}

// u128 x u64 -> u128 (the product must fit).
__host__ __device__ __forceinline__ u128 mul128x64(u128 a, u64 b) {
  const u64 lo = (u64)a;
  return ((u128)mulhi(lo, b) << 64 | (u128)(lo * b)) + ((u128)((u64)(a >> 64) * b) << 64);
}

// ---------------------------------------------------------------------------
// Gadget decomposition (prim/encryption/gadget.rs:115-190).
// ---------------------------------------------------------------------------
struct Gadget {
  u64 base;
  int L;
  int c;          // digits taken from the low chunk (B^c < 2^62); L - c from the high
  u128 S;         // B^L
  u64 Bc;         // B^c
  double dBc, dS_over_Q, dQ;
  u128 Q, halfQ;
  u64 half_base;
  u64 magic;      // floor(2^64 / B) for the 64-bit digit divisions
  bool small;     // Q * (S + 1) < 2^53: one limb, and the scaling is exact in doubles
  // Exact integer scaling round(|c| S / Q):
  //  mode 0: one modulus Q < 2^64 with Q * S < 2^127: num = |c| S + floor(Q/2)
  //          fits 128 bits, one 128-by-64 division by Q;
  //  mode 1: Q = q0 * q1 (RNS) with S * max(q0, q1) < 2^127: c = a0 + q0 t, and
  //          floor(num / Q) = floor((floor((a0 S + floor(Q/2)) / q0) + t S) / q1),
  //          two 128-by-64 divisions (exact: the remainder of the first division
  //          is below q0 and cannot carry into the second quotient);
  //  mode 2: otherwise, the double-precision estimate with exact fix-ups.
  int mode;
  Div64 dq, dq1;  // mode 0: Q; mode 1: q0 and q1
  u64 q0, q1;     // mode 1 limbs
  Div64 dbc;      // B^c, for the two-chunk split when S >= 2^64
  // Digit extraction in 32-bit pieces of c32 digits (B^c32 < 2^32).
  int c32;
  Div64 dc32;     // B^c32
  u32 bmagic;     // floor((2^32 - 1) / B)
};

inline Gadget make_gadget(u64 base, int L, u128 Q, u64 q0 = 0, u64 q1 = 0) {
  Gadget g{};
  g.base = base;
  g.L = L;
  u128 S = 1;
  int c = 0;
  u128 Bc = 1;
  for (int i = 0; i < L; ++i) {
    if ((long double)S * base >= 1.7e38L) throw CudaError(100, "gadget: B^L exceeds 2^127");
    S *= base;
    if (S < ((u128)1 << 62)) {
      c = i + 1;
      Bc = S;
    }
  }
  // The high chunk holds L - c digits plus a carry; it must fit 62 bits.
  u128 hi = 1;
  for (int i = c; i < L; ++i) hi *= base;
  if (hi >= ((u128)1 << 62)) throw CudaError(100, "gadget: B^L too large for two chunks");
  g.c = c;
  g.S = S;
  g.Bc = (u64)Bc;
  g.dBc = (double)(u64)Bc;
  g.Q = Q;
  g.halfQ = Q / 2;
  g.dQ = (double)(u64)(Q >> 64) * 18446744073709551616.0 + (double)(u64)Q;
  double dS = (double)(u64)(S >> 64) * 18446744073709551616.0 + (double)(u64)S;
  g.dS_over_Q = dS / g.dQ;
  g.half_base = base / 2;
  g.magic = (u64)(((u128)1 << 64) / base);
  g.small = Q < ((u128)1 << 53) && S < ((u128)1 << 53) && Q * (S + 1) < ((u128)1 << 53);
  // Exact integer scaling mode (see the struct). (long double) products only
  // decide the mode; the arithmetic itself is exact.
  const long double lS = (long double)(u64)(S >> 64) * 18446744073709551616.0L + (long double)(u64)S;
  const long double lQ = (long double)(u64)(Q >> 64) * 18446744073709551616.0L + (long double)(u64)Q;
  const long double two127 = 170141183460469231731687303715884105728.0L;
  if ((Q >> 64) == 0 && lQ * (lS + 1) < two127) {
    g.mode = 0;
    g.dq = make_div64((u64)Q);
  } else if (q0 && q1 && (u128)q0 * q1 == Q && lS * (long double)(q0 > q1 ? q0 : q1) * 2 < two127) {
    g.mode = 1;
    g.q0 = q0;
    g.q1 = q1;
    g.dq = make_div64(q0);
    g.dq1 = make_div64(q1);
  } else {
    g.mode = 2;
  }
  if (c < L) g.dbc = make_div64((u64)Bc);
  int c32 = 0;
  u64 b32 = 1;
  while (c32 < L && (u128)b32 * base < ((u128)1 << 32)) {
    b32 *= base;
    ++c32;
  }
  g.c32 = c32;
  g.dc32 = make_div64(b32);
  g.bmagic = (u32)(0xFFFFFFFFull / base);
  return g;
}

// The gadget of a ring: Q and (for a two-prime RNS ring) its limbs.
inline Gadget make_gadget(u64 base, int L, const DevRing& R) {
  return R.nl == 2 ? make_gadget(base, L, R.Q(), R.m[0].q, R.m[1].q) : make_gadget(base, L, R.Q());
}

// u / B and u % B for u < 2^63 via a reciprocal and a fix-up.
__host__ __device__ __forceinline__ u64 divB(u64 u, const Gadget& g, u64& rem) {
  u64 q = mulhi(u, g.magic);
  u64 r = u - q * g.base;
  for (int it = 0; it < 4 && r >= g.base; ++it) {
    r -= g.base;
    ++q;
  }
  rem = r;
  return q;
}

// Extract `cnt` balanced digits of u (LSB first) into d[]; returns the carry-out.
__host__ __device__ __forceinline__ u64 digits64(u64 u, int cnt, const Gadget& g, i64* d) {
  for (int k = 0; k < cnt; ++k) {
    u64 r;
    u64 q = divB(u, g, r);
    if (r > g.half_base) {
      d[k] = (i64)r - (i64)g.base;
      u = q + 1;
    } else {
      d[k] = (i64)r;
      u = q;
    }
  }
  return u;
}

// floor(n / d) for a 64-bit n.
__host__ __device__ __forceinline__ u64 div64by64(u64 n, const Div64& D, u64& rem) {
  const int s = D.s;
  const u64 n1 = s ? n >> (64 - s) : 0, n0 = n << s;
  u64 r;
  const u64 q = div_2by1(n1, n0, D, r);
  rem = r >> s;
  return q;
}

// The scaled value of one coefficient reduced mod B^L into [0, B^L): the
// centred lift c (v <= Q/2 ? v : v - Q), then round(|c| B^L / Q) =
// floor((|c| B^L + floor(Q/2)) / Q) with c's sign (gadget.rs:115-151,
// wide.rs:145-153). The balanced digits (gadget.rs:168-190) depend only on
// this value mod B^L.
// A `small` gadget (one limb, Q (S + 1) < 2^53) has a 64-bit numerator and a
// result below S < 2^53, the single digit chunk.
__host__ __device__ __forceinline__ u64 gadget_scaled_small(u64 a0, const Gadget& g) {
  const u64 Q = (u64)g.Q, hq = (u64)g.halfQ, S = (u64)g.S;
  const bool neg = a0 > hq;
  const u64 mag = neg ? Q - a0 : a0;
  u64 r;
  const u64 qe = div64by64(mag * S + hq, g.dq, r);
  return (neg && qe != 0) ? S - qe : qe;
}

// Mode 2 (large single-limb moduli): a double-precision quotient estimate and
// exact integer fix-ups.
__host__ __device__ __forceinline__ u128 gadget_scaled_fp(u128 v, const Gadget& g) {
  bool neg = v > g.halfQ;
  u128 mag = neg ? g.Q - v : v;
  u128 qe = double_to_u128(u128_to_double(mag) * g.dS_over_Q);
  i128 r = (i128)(mag * g.S + g.halfQ - qe * g.Q);
  i128 qc = (i128)(i64)floor(i128_to_double(r) / g.dQ);
  r -= qc * (i128)g.Q;
  qe = (u128)((i128)qe + qc);
  for (int it = 0; it < 4 && r < 0; ++it) {
    r += (i128)g.Q;
    qe -= 1;
  }
  for (int it = 0; it < 4 && r >= (i128)g.Q; ++it) {
    r -= (i128)g.Q;
    qe += 1;
  }
  return (neg && qe != 0) ? g.S - qe : qe;
}

__host__ __device__ __forceinline__ u128 gadget_scaled(u64 a0, u64 a1, const DevRing& R, const Gadget& g) {
  if (g.small) return (u128)gadget_scaled_small(a0, g);
  if (g.mode == 1) {
    // c = a0 + q0 t with the CRT digit t = (a1 - a0) q0^-1 mod q1.
    const DevMod& m1 = R.m[1];
    const u64 t = mul_shoup(submod(a1, reduce64(a0, m1), m1.q), R.q0inv_mod_q1, R.q0inv_shoup, m1.q);
    const u128 c = (u128)a0 + (u128)g.q0 * t;
    const bool neg = c > g.halfQ;
    // |c| = a + q0 u in the same mixed radix.
    u64 a = a0, u = t;
    if (neg) {
      a = a0 ? g.q0 - a0 : 0;
      u = a0 ? g.q1 - 1 - t : g.q1 - t;
    }
    u64 rem;
    const u128 x1 = div128by64(mul128x64(g.S, a) + g.halfQ, g.dq, rem);
    const u128 qe = div128by64(x1 + mul128x64(g.S, u), g.dq1, rem);
    return (neg && qe != 0) ? g.S - qe : qe;
  }
  const u128 v = R.nl == 2 ? crt2(a0, a1, R) : (u128)a0;
  if (g.mode == 0) {
    const bool neg = v > g.halfQ;
    const u64 mag = (u64)(neg ? g.Q - v : v);
    u64 rem;
    const u128 qe = div128by64(mul128x64(g.S, mag) + g.halfQ, g.dq, rem);
    return (neg && qe != 0) ? g.S - qe : qe;
  }
  return gadget_scaled_fp(v, g);
}

// Splits the scaled value into the two 64-bit chunks the digit loop consumes:
// lo < B^c holds digits 0..c-1, hi holds digits c..L-1 (plus lo's carry).
__host__ __device__ __forceinline__ void gadget_chunks(u128 u, const Gadget& g, u64& lo, u64& hi) {
  if (g.c >= g.L) {
    lo = (u64)u;
    hi = 0;
  } else {
    u64 rem;
    hi = (u64)div128by64(u, g.dbc, rem);
    lo = rem;
  }
}

// Next balanced digit (k-th, LSB first) from the running chunk value `cur`;
// at k == c the high chunk takes over with the low chunk's carry.
__host__ __device__ __forceinline__ i64 gadget_next_digit(u64& cur, u64 hi, int k, const Gadget& g) {
  if (k == g.c) cur = hi + cur;
  u64 r;
  u64 q = divB(cur, g, r);
  if (r > g.half_base) {
    cur = q + 1;
    return (i64)r - (i64)g.base;
  }
  cur = q;
  return (i64)r;
}

// Next balanced digit of a single-chunk (small) gadget.
__host__ __device__ __forceinline__ i64 gadget_next_digit_small(u64& cur, const Gadget& g) {
  u64 r;
  u64 q = divB(cur, g, r);
  if (r > g.half_base) {
    cur = q + 1;
    return (i64)r - (i64)g.base;
  }
  cur = q;
  return (i64)r;
}

__host__ __device__ __forceinline__ u32 mulhi32(u32 a, u32 b) {
#ifdef __CUDA_ARCH__
  return __umulhi(a, b);
#else
  return (u32)(((u64)a * b) >> 32);
#endif
}

// The balanced base-B digits of a scaled value v < B^L, LSB first, passed to
// f(k, d). v is cut into 32-bit pieces of c32 digits (one 128-by-64 division
// per piece but the last); each piece plus the carry of the previous one
// (at most B^c32 < 2^32) yields its digits with 32-bit divisions by B. The
// carry out of the top digit is dropped (the digits depend on v mod B^L).
template <class F>
__host__ __device__ __forceinline__ void for_each_digit(u128 v, const Gadget& g, F&& f) {
  const u32 B = (u32)g.base, half = (u32)g.half_base;
  u32 carry = 0;
  for (int k = 0; k < g.L;) {
    u32 x;
    if (k + g.c32 < g.L) {
      u64 rem;
      v = div128by64(v, g.dc32, rem);
      x = (u32)rem + carry;
    } else {
      x = (u32)v + carry;
    }
    const int cnt = g.L - k < g.c32 ? g.L - k : g.c32;
    for (int i = 0; i < cnt; ++i, ++k) {
      u32 q = mulhi32(x, g.bmagic);  // floor(x / B) - {0, 1, 2}
      u64 r = (u64)x - (u64)q * B;
      if (r >= B) {
        r -= B;
        ++q;
      }
      if (r >= B) {
        r -= B;
        ++q;
      }
      if (r > half) {
        f(k, (i64)r - (i64)B);
        x = q + 1;
      } else {
        f(k, (i64)r);
        x = q;
      }
    }
    carry = x;
  }
}

// The next balanced digit of a running 32-bit value x < 2^32 (LSB first).
__host__ __device__ __forceinline__ i64 gadget_next_digit32(u32& x, const Gadget& g) {
  const u32 B = (u32)g.base;
  u32 q = mulhi32(x, g.bmagic);
  u64 r = (u64)x - (u64)q * B;
  if (r >= B) {
    r -= B;
    ++q;
  }
  if (r >= B) {
    r -= B;
    ++q;
  }
  if (r > g.half_base) {
    x = q + 1;
    return (i64)r - (i64)B;
  }
  x = q;
  return (i64)r;
}

// Digits of one coefficient given its residues (nl limbs). Writes L signed
// digits, d[k] = k-th least significant (pairs with sample L-1-k).
__host__ __device__ inline void decompose_coeff(u64 a0, u64 a1, const DevRing& R, const Gadget& g, i64* d) {
  for_each_digit(gadget_scaled(a0, a1, R, g), g, [&](int k, i64 v) { d[k] = v; });
}

}  // namespace via
