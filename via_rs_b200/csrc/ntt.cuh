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
};

// Host owner of the device tables of one prime.
struct NttTableHost {
  NttTable dev{};
  u64* buf = nullptr;
  bool valid = false;
};

// One phase (up to three butterfly stages) of the register-resident transform:
// each thread holds 8 residues of a length-2^LOGN segment. Stage s of the
// forward transform pairs (x, x + len_s), len_s = n >> (s+1), with twiddle
// psi[n/(2 len_s) + x/(2 len_s)] (Cooley-Tukey, bit-reversed twiddles); the
// inverse runs len = 1, 2, ..., n/2 (Gentleman-Sande, psi^-1). Phase P covers
// stages 3P..3P+R-1 and works on sub-blocks of 2^R residues x = base + k*STRIDE,
// where STRIDE is the phase's smallest len and base = (u / STRIDE) *
// (STRIDE << R) + u % STRIDE over the n >> R sub-blocks u; a thread owns
// 8 >> R consecutive sub-blocks.
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
      const int base = (u / STRIDE) * (STRIDE << R) + (u % STRIDE);
#pragma unroll
      for (int lvl = 0; lvl < R; ++lvl) {
        // forward: len = STRIDE << (R-1-lvl) (decreasing); inverse: STRIDE << lvl.
        const int hk = INV ? (1 << lvl) : (1 << (R - 1 - lvl));
        const int len = STRIDE * hk;
        const int m = n / (2 * len);
#pragma unroll
        for (int k = 0; k < (1 << R); ++k) {
          if (k & hk) continue;
          const int x = base + k * STRIDE;
          const int grp = x / (2 * len);
          u64& a = e[sub * (1 << R) + k];
          u64& c = e[sub * (1 << R) + k + hk];
          if (!INV) {
            const u64 w = __ldg(T.psi + m + grp), ws = __ldg(T.psi_sh + m + grp);
            const u64 t = mul_shoup(c, w, ws, q);
            const u64 av = a;
            a = addmod(av, t, q);
            c = submod(av, t, q);
          } else {
            const u64 w = __ldg(T.ipsi + m + grp), ws = __ldg(T.ipsi_sh + m + grp);
            const u64 av = a, cv = c;
            a = addmod(av, cv, q);
            c = mul_shoup(submod(av, cv, q), w, ws, q);
          }
        }
      }
    }
  }
};


// Forward transform of a segment whose residues a thread already holds in the
// phase-0 layout (NttPhase<LOGN,false,0>::index); leaves them in the layout of
// the last phase. `ssm` is the segment's n-residue shared-memory exchange area.
template <int LOGN, int P = 0>
__device__ __forceinline__ void ntt_forward_regs(u64 (&e)[8], int tid, const NttTable& T, u64* ssm) {
  using Ph = NttPhase<LOGN, false, P>;
  constexpr int NPH = (LOGN + 2) / 3;
  Ph::run(e, tid, T);
  if constexpr (P + 1 < NPH) {
    using Nx = NttPhase<LOGN, false, P + 1>;
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) ssm[Ph::index(v, tid)] = e[v];
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) e[v] = ssm[Nx::index(v, tid)];
    ntt_forward_regs<LOGN, P + 1>(e, tid, T, ssm);
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
    for (int v = 0; v < 8; ++v) ssm[Ph::index(v, tid)] = e[v];
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) e[v] = ssm[Nx::index(v, tid)];
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

}  // namespace via
