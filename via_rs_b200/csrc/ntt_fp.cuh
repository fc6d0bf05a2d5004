// The register-resident negacyclic transform of ntt.cuh in double precision,
// for single primes q < 2^36. Residues are integer-valued doubles in a signed
// range, and every product is exact:
//
//   fp_mulmod(a, b): ph = fl(a b), pl = a b - ph (one FMA: the error-free
//   product), qt = round(ph / q) (an FMA against a rounded 1/q plus the
//   1.5 * 2^52 rounding constant), r = (ph - qt q) + pl.
//
// For integers |a| < 2^48 and |b| < q, |qt - a b / q| <= 1/2 + 2^-4, so
// ph - qt q and r are integers far below 2^53 and both steps are exact:
// r = a b (mod q) with |r| <= 0.5625 q (checked against 128-bit integer
// products over these ranges). This is the floating-point reduction of
// modular products used by Shoup's NTL (a quotient estimate in floating point,
// an exact integer correction), with the FMA two-product making the product
// itself exact. Explicit _rn intrinsics keep the compiler from contracting or
// reassociating any step.
//
// Bounds (q < 2^36, n <= 4096): forward butterflies (a, c) -> (a + t, a - t),
// t = fp_mulmod(c, w), grow by at most 0.5625 q per stage; inverse butterflies
// (a, c) -> (a + c, fp_mulmod(a - c, w)) at most double per stage, so inputs
// below q stay below 2^12 q < 2^48 after twelve stages. The inverse ends with
// an fp_mulmod by n^-1.
#pragma once
#include "ntt.cuh"

namespace via {

constexpr double FP_ROUND = 6755399441055744.0;  // 1.5 * 2^52: x + FP_ROUND - FP_ROUND rounds x to an integer

__device__ __forceinline__ double fp_mulmod(double a, double b, double q, double qinv) {
  const double ph = __dmul_rn(a, b);
  const double pl = __fma_rn(a, b, -ph);
  const double qt = __dadd_rn(__fma_rn(ph, qinv, FP_ROUND), -FP_ROUND);
  return __dadd_rn(__fma_rn(-qt, q, ph), pl);
}

// Signed residue x (|x| < 2^50) -> canonical residue in [0, q).
__device__ __forceinline__ double fp_canonical(double x, double q, double qinv) {
  const double qt = __dadd_rn(__fma_rn(x, qinv, FP_ROUND), -FP_ROUND);
  double r = __fma_rn(-qt, q, x);  // exact, |r| <= q / 2 + 1
  if (r < 0) r = __dadd_rn(r, q);
  if (r >= q) r = __dadd_rn(r, -q);
  return r;
}

// One phase of the transform: the butterflies of NttPhase<LOGN, INV, P> on
// doubles, with the same sub-block layout (NttPhase::index).
template <int LOGN, bool INV, int P>
struct NttPhaseFp {
  using Ix = NttPhase<LOGN, INV, P>;
  static constexpr int n = Ix::n, S0 = Ix::S0, R = Ix::R, NSUB = Ix::NSUB, STRIDE = Ix::STRIDE;

  __device__ __forceinline__ static void run(double (&e)[8], int tid, const NttTable& T) {
    const double q = T.qd, qinv = T.qinv;
#pragma unroll
    for (int sub = 0; sub < NSUB; ++sub) {
      const int u = tid * NSUB + sub;
      const int b0 = u / STRIDE;
#pragma unroll
      for (int lvl = 0; lvl < R; ++lvl) {
        const int hk = INV ? (1 << lvl) : (1 << (R - 1 - lvl));
        const int len = STRIDE * hk;
        const int m = n / (2 * len);
        const int tw0 = m + (INV ? (b0 << (R - 1 - lvl)) : (b0 << lvl));
        double w[4];
        const int ntw = INV ? (1 << (R - 1 - lvl)) : (1 << lvl);
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (j < ntw) w[j] = __ldg((INV ? T.ipsi_d : T.psi_d) + tw0 + j);
#pragma unroll
        for (int k = 0; k < (1 << R); ++k) {
          if (k & hk) continue;
          const int j = INV ? (k >> (lvl + 1)) : (k >> (R - lvl));
          double& a = e[sub * (1 << R) + k];
          double& c = e[sub * (1 << R) + k + hk];
          if (!INV) {
            const double t = fp_mulmod(c, w[j], q, qinv);
            const double av = a;
            a = __dadd_rn(av, t);
            c = __dadd_rn(av, -t);
          } else {
            const double av = a, cv = c;
            a = __dadd_rn(av, cv);
            c = fp_mulmod(__dadd_rn(av, -cv), w[j], q, qinv);
          }
        }
      }
    }
  }
};

// Forward transform of a segment held in the phase-0 layout; leaves it in the
// layout of the last phase, as signed residues below |input| + 0.5625 LOGN q.
template <int LOGN, int P = 0>
__device__ __forceinline__ void ntt_forward_fp(double (&e)[8], int tid, const NttTable& T, double* ssm) {
  using Ph = NttPhaseFp<LOGN, false, P>;
  constexpr int NPH = (LOGN + 2) / 3;
  Ph::run(e, tid, T);
  if constexpr (P + 1 < NPH) {
    using Nx = NttPhase<LOGN, false, P + 1>;
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) ssm[swz(Ph::Ix::index(v, tid))] = e[v];
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) e[v] = ssm[swz(Nx::index(v, tid))];
    ntt_forward_fp<LOGN, P + 1>(e, tid, T, ssm);
  }
}

// Inverse transform (then the n^-1 scaling) of a segment held in the layout
// NttPhase<LOGN, true, 0>::index, inputs below 4 q in magnitude; leaves signed
// coefficients, |x| <= 0.5625 q, in the layout of the last inverse phase. With
// REDUCE (needed for q above 2^35) every phase boundary first brings the values
// back within q/2, so a phase of three stages stays below 32 q.
template <int LOGN, int P = 0, bool REDUCE = false>
__device__ __forceinline__ void ntt_inverse_fp(double (&e)[8], int tid, const NttTable& T, double* ssm) {
  using Ph = NttPhaseFp<LOGN, true, P>;
  constexpr int NPH = (LOGN + 2) / 3;
  Ph::run(e, tid, T);
  if constexpr (P + 1 < NPH) {
    using Nx = NttPhase<LOGN, true, P + 1>;
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) ssm[swz(Ph::Ix::index(v, tid))] = e[v];
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) e[v] = ssm[swz(Nx::index(v, tid))];
    if constexpr (REDUCE) {
#pragma unroll
      for (int v = 0; v < 8; ++v)
        e[v] = __fma_rn(-__dadd_rn(__fma_rn(e[v], T.qinv, FP_ROUND), -FP_ROUND), T.qd, e[v]);
    }
    ntt_inverse_fp<LOGN, P + 1, REDUCE>(e, tid, T, ssm);
  } else {
#pragma unroll
    for (int v = 0; v < 8; ++v) e[v] = fp_mulmod(e[v], T.ninv_d[LOGN], T.qd, T.qinv);
  }
}

}  // namespace via
