// Batched negacyclic NTT over one or two primes (the eval form of a ring
// element). The reference's eval form (crates/via-primitives/src/algebra/ring/
// ntt.rs:305-425) never leaves the server, so this build uses its own root and
// ordering; only coefficient-form results are observable and they are exact.
#pragma once
#include <vector>

#include "common.cuh"

namespace via {

constexpr int NTT_MAX_LOGN = 12;  // n <= 4096

// Device view of one prime's tables. psi[k] = psi^bitrev(k) for k < nmax; the
// prefix of length n is the table of the degree-n transform (bitrev over
// log2(nmax) bits of k < n equals bitrev over log2(n) bits times nmax/n).
struct NttTable {
  u64 q;
  int nmax;
  int pad;
  const u64* psi;      // forward twiddles
  const u64* psi_sh;   // their Shoup constants
  const u64* ipsi;     // inverse twiddles
  const u64* ipsi_sh;
  u64 ninv[NTT_MAX_LOGN + 1];
  u64 ninv_sh[NTT_MAX_LOGN + 1];
  // The same twiddles as exact doubles (q < 2^50), for the double-precision
  // transforms of ntt_fp.cuh.
  const double* psi_d;
  const double* ipsi_d;
  double qd, qinv;  // q and a rounded 1 / q
  double ninv_d[NTT_MAX_LOGN + 1];
};

// Host owner of the device tables of one prime.
struct NttTableHost {
  NttTable dev{};
  u64* buf = nullptr;
  bool valid = false;
};

// Shoup product without the final correction: a * w mod q in [0, 2q) for any
// a < 2^64 (w < q, ws = floor(w * 2^64 / q)).
__device__ __forceinline__ u64 shoup_lazy(u64 a, u64 w, u64 ws, u64 q) { return a * w - mulhi(a, ws) * q; }

// Shared-memory slot of element x of an exchange: an XOR swizzle of the low
// four bits by bits 4..9 keeps the strided phase layouts free of 8-byte bank
// conflicts (at most two lanes of a half warp per bank). A bijection on every
// aligned 16-element block, so segments of n >= 16 stay in place.
__device__ __forceinline__ int swz(int x) { return x ^ (((x >> 4) ^ (x >> 5)) & 15); }

// One phase (up to three butterfly stages) of the register-resident transform:
// each thread holds 8 residues of a length-2^LOGN segment. Stage s of the
// forward transform pairs (x, x + len_s), len_s = n >> (s+1), with twiddle
// psi[n/(2 len_s) + x/(2 len_s)] (Cooley-Tukey, bit-reversed twiddles); the
// inverse runs len = 1, 2, ..., n/2 (Gentleman-Sande, psi^-1). Phase P covers
// stages 3P..3P+R-1 and works on sub-blocks of 2^R residues x = base + k*STRIDE,
// where STRIDE is the phase's smallest len and base = (u / STRIDE) *
// (STRIDE << R) + u % STRIDE over the n >> R sub-blocks u; a thread owns
// 8 >> R consecutive sub-blocks. A sub-block's butterflies at level lvl use
// 2^lvl (forward) or 2^(R-1-lvl) (inverse) consecutive twiddles starting at
// (u / STRIDE) times that count.
//
// Lazy residues (no conditional corrections inside a transform):
//  * forward: t = a*w mod q in [0, 2q); (a, c) -> (a + t, a + 2q - t), so after
//    s stages every residue is below (1 + 2s) q;
//  * inverse: stage s inputs are below 2^s q; (a, c) -> (a + c, (a + 2^s q - c) w
//    mod q in [0, 2q)).
// Both stay far below 2^64 for q < 2^50 and n <= 4096; the transforms end
// with one exact reduction (forward) or the n^-1 scaling (inverse).
template <int LOGN, bool INV, int P>
struct NttPhase {
  static constexpr int n = 1 << LOGN;
  static constexpr int S0 = 3 * P;
  static constexpr int R = (LOGN - S0) < 3 ? (LOGN - S0) : 3;
  static constexpr int NSUB = 8 >> R;
  // Smallest stage len of the phase (see k_ntt_reg).
  static constexpr int STRIDE = INV ? (1 << S0) : ((n >> (S0 + 1)) >> (R - 1));

  __device__ __forceinline__ static int index(int v, int tid) {
    const int sub = v >> R, k = v & ((1 << R) - 1);
    const int u = tid * NSUB + sub;
    return (u / STRIDE) * (STRIDE << R) + (u % STRIDE) + k * STRIDE;
  }

  __device__ __forceinline__ static void run(u64 (&e)[8], int tid, const NttTable& T) {
    const u64 q = T.q;
#pragma unroll
    for (int sub = 0; sub < NSUB; ++sub) {
      const int u = tid * NSUB + sub;
      const int b0 = u / STRIDE;
#pragma unroll
      for (int lvl = 0; lvl < R; ++lvl) {
        // forward: len = STRIDE << (R-1-lvl) (decreasing); inverse: STRIDE << lvl.
        const int hk = INV ? (1 << lvl) : (1 << (R - 1 - lvl));
        const int len = STRIDE * hk;
        const int m = n / (2 * len);
        const int tw0 = m + (INV ? (b0 << (R - 1 - lvl)) : (b0 << lvl));
        u64 w[4], ws[4];
        const int ntw = INV ? (1 << (R - 1 - lvl)) : (1 << lvl);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (j < ntw) {
            w[j] = __ldg((INV ? T.ipsi : T.psi) + tw0 + j);
            ws[j] = __ldg((INV ? T.ipsi_sh : T.psi_sh) + tw0 + j);
          }
        }
#pragma unroll
        for (int k = 0; k < (1 << R); ++k) {
          if (k & hk) continue;
          const int j = INV ? (k >> (lvl + 1)) : (k >> (R - lvl));
          u64& a = e[sub * (1 << R) + k];
          u64& c = e[sub * (1 << R) + k + hk];
          if (!INV) {
            const u64 t = shoup_lazy(c, w[j], ws[j], q);
            const u64 av = a;
            a = av + t;
            c = av + 2 * q - t;
          } else {
            const u64 av = a, cv = c;
            a = av + cv;
            c = shoup_lazy(av + (q << (S0 + lvl)) - cv, w[j], ws[j], q);
          }
        }
      }
    }
  }
};

// Exact residue of a lazy forward output (below 2^64): Shoup by 1.
__device__ __forceinline__ u64 ntt_canonical(u64 x, const NttTable& T) {
  return mul_shoup(x, T.ninv[0], T.ninv_sh[0], T.q);
}

// Forward transform of a segment whose residues a thread already holds in the
// phase-0 layout (NttPhase<LOGN,false,0>::index); leaves them (exact) in the
// layout of the last phase. `ssm` is an n-residue shared-memory exchange area
// of one segment, addressed through swz().
// With LAZY the outputs stay below (1 + 2 LOGN) q instead of being reduced,
// for callers that reduce a sum of products once at the end.
template <int LOGN, int P = 0, bool LAZY = false>
__device__ __forceinline__ void ntt_forward_regs(u64 (&e)[8], int tid, const NttTable& T, u64* ssm) {
  using Ph = NttPhase<LOGN, false, P>;
  constexpr int NPH = (LOGN + 2) / 3;
  Ph::run(e, tid, T);
  if constexpr (P + 1 < NPH) {
    using Nx = NttPhase<LOGN, false, P + 1>;
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) ssm[swz(Ph::index(v, tid))] = e[v];
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) e[v] = ssm[swz(Nx::index(v, tid))];
    ntt_forward_regs<LOGN, P + 1, LAZY>(e, tid, T, ssm);
  } else if constexpr (!LAZY) {
#pragma unroll
    for (int v = 0; v < 8; ++v) e[v] = ntt_canonical(e[v], T);
  }
}

// Inverse transform (Gentleman-Sande, then the n^-1 scaling) of a segment whose
// eval-form residues a thread holds in the layout NttPhase<LOGN,true,0>::index;
// leaves the coefficients in the layout of the last inverse phase.
template <int LOGN, int P = 0>
__device__ __forceinline__ void ntt_inverse_regs(u64 (&e)[8], int tid, const NttTable& T, u64* ssm) {
  using Ph = NttPhase<LOGN, true, P>;
  constexpr int NPH = (LOGN + 2) / 3;
  Ph::run(e, tid, T);
  if constexpr (P + 1 < NPH) {
    using Nx = NttPhase<LOGN, true, P + 1>;
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) ssm[swz(Ph::index(v, tid))] = e[v];
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) e[v] = ssm[swz(Nx::index(v, tid))];
    ntt_inverse_regs<LOGN, P + 1>(e, tid, T, ssm);
  } else {
#pragma unroll
    for (int v = 0; v < 8; ++v) e[v] = mul_shoup(e[v], T.ninv[LOGN], T.ninv_sh[LOGN], T.q);
  }
}

// Builds tables for q (prime, 2*nmax | q-1). Returns valid=false otherwise.
NttTableHost make_ntt_table(u64 q, int nmax);
void free_ntt_table(NttTableHost& t);
bool is_ntt_friendly(u64 q, int n);

// In-place transforms of `segments` consecutive length-n segments starting at
// `data`; segment s uses table (s % nl == 0 ? t0 : t1) (limb-major polys).
void ntt_forward(u64* data, int n, int nl, long segments, const NttTable& t0, const NttTable& t1,
                 cudaStream_t st);
void ntt_inverse(u64* data, int n, int nl, long segments, const NttTable& t0, const NttTable& t1,
                 cudaStream_t st);
// Forward transform whose outputs are left below (1 + 2 log2 n) q (n >= 8;
// n = 2, 4 give exact residues), for operands of a 128-bit sum of products.
void ntt_forward_lazy(u64* data, int n, int nl, long segments, const NttTable& t0, const NttTable& t1,
                      cudaStream_t st);
// The same from signed 8-bit digit polynomials: segment s (limb s % nl of
// polynomial s / nl) reads din + (s / nl) * n and writes out + s * n.
void ntt_forward_i8_lazy(const int8_t* din, u64* out, int n, int nl, long segments, const NttTable& t0,
                         const NttTable& t1, cudaStream_t st);
// The same with signed double outputs (within 0.5625 log2(n) q + 127 of zero,
// exact integers), for the double-precision multiply-accumulates; primes below 2^44.
void ntt_forward_i8_fp(const int8_t* din, double* out, int n, int nl, long segments, const NttTable& t0,
                       const NttTable& t1, cudaStream_t st);
// Whether the double-precision transforms serve these primes (both below 2^44).
bool ntt_fp_ok(const NttTable& t0, const NttTable& t1);

}  // namespace via
