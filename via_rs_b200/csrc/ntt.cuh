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
