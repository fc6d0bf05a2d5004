// Batched negacyclic NTT kernels (shared-memory staged, radix-2, Shoup twiddles).
#include <algorithm>
#include <cstring>

#include "ntt.cuh"
#include "ntt_fp.cuh"

namespace via {

static u64 h_mulmod(u64 a, u64 b, u64 q) { return (u64)((u128)a * b % q); }
static u64 h_pow(u64 b, u64 e, u64 q) {
  u64 r = 1 % q;
  b %= q;
  while (e) {
    if (e & 1) r = h_mulmod(r, b, q);
    b = h_mulmod(b, b, q);
    e >>= 1;
  }
  return r;
}
static bool h_is_prime(u64 n) {
  if (n < 2) return false;
  for (u64 p : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull})
    if (n % p == 0) return n == p;
  u64 d = n - 1;
  int s = 0;
  while (!(d & 1)) {
    d >>= 1;
    ++s;
  }
  for (u64 a : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
    u64 x = h_pow(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int r = 1; r < s; ++r) {
      x = h_mulmod(x, x, n);
      if (x == n - 1) {
        comp = false;
        break;
      }
    }
    if (comp) return false;
  }
  return true;
}

bool is_ntt_friendly(u64 q, int n) {
  return n >= 2 && (q & (q - 1)) != 0 && q < (1ull << 62) && (q - 1) % (2 * (u64)n) == 0 && h_is_prime(q);
}

static int bitrev(int x, int logn) {
  int r = 0;
  for (int i = 0; i < logn; ++i) r |= ((x >> i) & 1) << (logn - 1 - i);
  return r;
}

NttTableHost make_ntt_table(u64 q, int nmax) {
  NttTableHost h;
  if (!is_ntt_friendly(q, nmax)) return h;
  u64 psi = 0;
  for (u64 g = 2; g < q; ++g) {
    u64 c = h_pow(g, (q - 1) / (2 * (u64)nmax), q);
    if (h_pow(c, (u64)nmax, q) == q - 1) {
      psi = c;
      break;
    }
  }
  int logn = __builtin_ctz((unsigned)nmax);
  u64 ipsi = h_pow(psi, q - 2, q);
  std::vector<u64> host(6 * (size_t)nmax);
  for (int k = 0; k < nmax; ++k) {
    u64 w = h_pow(psi, (u64)bitrev(k, logn), q);
    u64 wi = h_pow(ipsi, (u64)bitrev(k, logn), q);
    host[k] = w;
    host[nmax + k] = (u64)(((u128)w << 64) / q);
    host[2 * nmax + k] = wi;
    host[3 * nmax + k] = (u64)(((u128)wi << 64) / q);
    const double wd = (double)w, wid = (double)wi;  // exact: w, wi < q < 2^50
    std::memcpy(&host[4 * nmax + k], &wd, 8);
    std::memcpy(&host[5 * nmax + k], &wid, 8);
  }
  VIA_CUDA(cudaMalloc(&h.buf, host.size() * 8));
  VIA_CUDA(cudaMemcpy(h.buf, host.data(), host.size() * 8, cudaMemcpyHostToDevice));
  h.dev.q = q;
  h.dev.nmax = nmax;
  h.dev.psi = h.buf;
  h.dev.psi_sh = h.buf + nmax;
  h.dev.ipsi = h.buf + 2 * nmax;
  h.dev.ipsi_sh = h.buf + 3 * nmax;
  h.dev.psi_d = reinterpret_cast<const double*>(h.buf + 4 * nmax);
  h.dev.ipsi_d = reinterpret_cast<const double*>(h.buf + 5 * nmax);
  h.dev.qd = (double)q;
  h.dev.qinv = 1.0 / (double)q;
  for (int l = 0; l <= NTT_MAX_LOGN; ++l) {
    u64 ninv = h_pow((u64)1 << l, q - 2, q);
    h.dev.ninv[l] = ninv;
    h.dev.ninv_sh[l] = (u64)(((u128)ninv << 64) / q);
    h.dev.ninv_d[l] = (double)ninv;
  }
  h.valid = true;
  return h;
}

void free_ntt_table(NttTableHost& t) {
  if (t.buf) cudaFree(t.buf);
  t.buf = nullptr;
  t.valid = false;
}

constexpr int NTT_THREADS = 256;

// ---------------------------------------------------------------------------
// Register-resident transform for n >= 8: every thread holds 8 residues and
// performs up to three butterfly stages (a radix-8 step) on them before the
// residues are exchanged through shared memory. A CTA of 256 threads handles
// 2048/n segments (one segment = one limb of one polynomial).
//
// Stage s of the forward transform pairs (x, x + len_s), len_s = n >> (s+1),
// twiddle psi[n/(2 len_s) + x/(2 len_s)] (Cooley-Tukey on bit-reversed twiddles);
// the inverse runs len = 1, 2, ..., n/2 with Gentleman-Sande butterflies and
// psi^-1, then scales by n^-1. A phase of r stages works on sub-blocks of 2^r
// residues x = base + k*stride, k < 2^r, where stride is the phase's smallest
// len and base = (u / stride) * (stride << r) + u % stride over the n >> r
// sub-blocks u; a thread owns 8 >> r consecutive sub-blocks.
// ---------------------------------------------------------------------------
// I8: the segment's input is a polynomial of signed 8-bit digits at `gin`,
// lifted into [0, q) on load; the output goes to g.
template <int LOGN, bool INV, int P, bool LAZY = false, bool I8 = false>
__device__ __forceinline__ void ntt_phases(u64 (&e)[8], int tid, const NttTable& T, u64* g, u64* sm, int sbase,
                                           bool active, const int8_t* gin = nullptr) {
  using Ph = NttPhase<LOGN, INV, P>;
  constexpr int NPH = (LOGN + 2) / 3;
  if (P == 0) {
    if constexpr (I8) {
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        const int d = active ? gin[Ph::index(v, tid)] : 0;
        e[v] = d >= 0 ? (u64)d : T.q - (u64)(-d);
      }
    } else {
#pragma unroll
      for (int v = 0; v < 8; ++v) e[v] = active ? g[Ph::index(v, tid)] : 0;
    }
  } else {
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) e[v] = sm[swz(sbase + Ph::index(v, tid))];
  }
  Ph::run(e, tid, T);
  if constexpr (P == NPH - 1) {
    if constexpr (INV || !LAZY) {
#pragma unroll
      for (int v = 0; v < 8; ++v)
        e[v] = INV ? mul_shoup(e[v], T.ninv[LOGN], T.ninv_sh[LOGN], T.q) : ntt_canonical(e[v], T);
    }
    if (active) {
#pragma unroll
      for (int v = 0; v < 8; ++v) g[Ph::index(v, tid)] = e[v];
    }
  } else {
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) sm[swz(sbase + Ph::index(v, tid))] = e[v];
    ntt_phases<LOGN, INV, P + 1, LAZY, false>(e, tid, T, g, sm, sbase, active);
  }
}

// Threads of one k_ntt_reg CTA: 256, or one segment's n/8 when that is more.
template <int LOGN>
__host__ __device__ constexpr int ntt_cta() {
  return ((1 << LOGN) / 8) > NTT_THREADS ? ((1 << LOGN) / 8) : NTT_THREADS;
}

// LAZY (forward only): outputs left below (1 + 2 LOGN) q, for digit transforms
// whose consumer reduces a 128-bit sum of products.
template <int LOGN, bool INV, bool LAZY = false>
__global__ void __launch_bounds__(ntt_cta<LOGN>()) k_ntt_reg(u64* __restrict__ data, int nl, long segments,
                                                             NttTable t0, NttTable t1) {
  constexpr int n = 1 << LOGN;
  constexpr int TPS = n / 8;                    // threads per segment
  constexpr int SPC = ntt_cta<LOGN>() / TPS;    // segments per CTA
  __shared__ u64 sm[ntt_cta<LOGN>() * 8];
  const int seg_local = threadIdx.x / TPS;
  const int tid = threadIdx.x % TPS;
  const long seg = (long)blockIdx.x * SPC + seg_local;
  const bool active = seg < segments;
  const NttTable& T = (nl == 2 && (seg & 1)) ? t1 : t0;
  u64 e[8];
  ntt_phases<LOGN, INV, 0, LAZY>(e, tid, T, data + seg * n, sm, seg_local * n, active);
}

// Lazy forward transforms of signed 8-bit digit polynomials: segment s (limb
// s % nl of digit polynomial s / nl) reads din + (s / nl) * n and writes
// out + s * n.
template <int LOGN>
__global__ void __launch_bounds__(ntt_cta<LOGN>()) k_ntt_reg_i8(const int8_t* __restrict__ din, u64* __restrict__ out,
                                                                int nl, long segments, NttTable t0, NttTable t1) {
  constexpr int n = 1 << LOGN;
  constexpr int TPS = n / 8;
  constexpr int SPC = ntt_cta<LOGN>() / TPS;
  __shared__ u64 sm[ntt_cta<LOGN>() * 8];
  const int seg_local = threadIdx.x / TPS;
  const int tid = threadIdx.x % TPS;
  const long seg = (long)blockIdx.x * SPC + seg_local;
  const bool active = seg < segments;
  const NttTable& T = (nl == 2 && (seg & 1)) ? t1 : t0;
  u64 e[8];
  ntt_phases<LOGN, false, 0, true, true>(e, tid, T, out + seg * n, sm, seg_local * n, active,
                                         din + (active ? seg / nl : 0) * n);
}

// ---------------------------------------------------------------------------
// The register-resident transforms in double precision (ntt_fp.cuh), for primes
// below 2^44: the same layouts and phases as ntt_phases, exact integer
// arithmetic on doubles. Inputs are residues below 2^47 (larger values are
// reduced first); outputs:
//  * forward: canonical residues, or (LAZY) nonnegative residues below
//    (1.125 LOGN + 3) q <= (1 + 2 LOGN) q, the integer kernel's lazy bound;
//    forward values stay within |input| + 0.5625 LOGN q of zero;
//  * inverse: canonical residues. Inverse values at most double per stage; for
//    q above 2^35 every phase boundary first reduces them to within q/2, so a
//    phase of three stages ends below 4 q and every product stays exact.
// I8: the input is a polynomial of signed 8-bit digits.
// ---------------------------------------------------------------------------
// DOUT: the (forward, lazy) outputs are stored as the signed doubles themselves.
template <int LOGN, bool INV, int P, bool LAZY, bool I8, bool DOUT = false>
__device__ __forceinline__ void ntt_fp_phases(double (&e)[8], int tid, const NttTable& T, u64* g, double* sm,
                                              int sbase, bool active, const int8_t* gin) {
  using Ph = NttPhaseFp<LOGN, INV, P>;
  using Ix = NttPhase<LOGN, INV, P>;
  constexpr int NPH = (LOGN + 2) / 3;
  const double q = T.qd, qinv = T.qinv;
  if constexpr (P == 0) {
    if constexpr (I8) {
#pragma unroll
      for (int v = 0; v < 8; ++v) e[v] = active ? (double)gin[Ix::index(v, tid)] : 0.0;
    } else {
#pragma unroll
      for (int v = 0; v < 8; ++v) {
        u64 x = active ? g[Ix::index(v, tid)] : 0;
        if (x >= (1ull << 47)) x %= T.q;
        e[v] = __ull2double_rn(x);
      }
    }
  } else {
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) e[v] = sm[swz(sbase + Ix::index(v, tid))];
    if (INV && q > 34359738368.0) {  // q > 2^35: restart the inverse's growth at q/2
#pragma unroll
      for (int v = 0; v < 8; ++v)
        e[v] = __fma_rn(-__dadd_rn(__fma_rn(e[v], qinv, FP_ROUND), -FP_ROUND), q, e[v]);
    }
  }
  Ph::run(e, tid, T);
  if constexpr (P == NPH - 1) {
    if constexpr (INV) {
#pragma unroll
      for (int v = 0; v < 8; ++v) e[v] = fp_canonical(fp_mulmod(e[v], T.ninv_d[LOGN], q, qinv), q, qinv);
    } else if constexpr (DOUT) {
      if (active) {
        double* gd = reinterpret_cast<double*>(g);
#pragma unroll
        for (int v = 0; v < 8; ++v) gd[Ix::index(v, tid)] = e[v];
      }
      return;
    } else if constexpr (LAZY) {
      constexpr int OFF = (9 * LOGN + 15) / 16 + 1;  // ceil(0.5625 LOGN) + 1
      const double off = (double)OFF * q;
#pragma unroll
      for (int v = 0; v < 8; ++v) e[v] = __dadd_rn(e[v], off);
    } else {
#pragma unroll
      for (int v = 0; v < 8; ++v) e[v] = fp_canonical(e[v], q, qinv);
    }
    if (active) {
#pragma unroll
      for (int v = 0; v < 8; ++v) g[Ix::index(v, tid)] = __double2ull_rn(e[v]);
    }
  } else {
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) sm[swz(sbase + Ix::index(v, tid))] = e[v];
    ntt_fp_phases<LOGN, INV, P + 1, LAZY, false, DOUT>(e, tid, T, g, sm, sbase, active, nullptr);
  }
}

template <int LOGN, bool INV, bool LAZY = false>
__global__ void __launch_bounds__(ntt_cta<LOGN>()) k_ntt_fp(u64* __restrict__ data, int nl, long segments,
                                                            NttTable t0, NttTable t1) {
  constexpr int n = 1 << LOGN;
  constexpr int TPS = n / 8;
  constexpr int SPC = ntt_cta<LOGN>() / TPS;
  __shared__ double sm[ntt_cta<LOGN>() * 8];
  const int seg_local = threadIdx.x / TPS;
  const int tid = threadIdx.x % TPS;
  const long seg = (long)blockIdx.x * SPC + seg_local;
  const bool active = seg < segments;
  const NttTable& T = (nl == 2 && (seg & 1)) ? t1 : t0;
  double e[8];
  ntt_fp_phases<LOGN, INV, 0, LAZY, false>(e, tid, T, data + seg * n, sm, seg_local * n, active, nullptr);
}

template <int LOGN, bool DOUT = false>
__global__ void __launch_bounds__(ntt_cta<LOGN>()) k_ntt_fp_i8(const int8_t* __restrict__ din, u64* __restrict__ out,
                                                               int nl, long segments, NttTable t0, NttTable t1) {
  constexpr int n = 1 << LOGN;
  constexpr int TPS = n / 8;
  constexpr int SPC = ntt_cta<LOGN>() / TPS;
  __shared__ double sm[ntt_cta<LOGN>() * 8];
  const int seg_local = threadIdx.x / TPS;
  const int tid = threadIdx.x % TPS;
  const long seg = (long)blockIdx.x * SPC + seg_local;
  const bool active = seg < segments;
  const NttTable& T = (nl == 2 && (seg & 1)) ? t1 : t0;
  double e[8];
  ntt_fp_phases<LOGN, false, 0, true, true, DOUT>(e, tid, T, out + seg * n, sm, seg_local * n, active,
                                                  din + (active ? seg / nl : 0) * n);
}

// n = 2 and 4 on 8-bit digits, double outputs: one thread per segment.
template <int LOGN>
__global__ void k_ntt_tiny_i8_fp(const int8_t* __restrict__ din, double* __restrict__ out, int nl, long segments,
                                 NttTable t0, NttTable t1) {
  constexpr int n = 1 << LOGN;
  long seg = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (seg >= segments) return;
  const NttTable& T = (nl == 2 && (seg & 1)) ? t1 : t0;
  double a[n];
  const int8_t* gi = din + (seg / nl) * n;
#pragma unroll
  for (int i = 0; i < n; ++i) a[i] = (double)gi[i];
#pragma unroll
  for (int len = n / 2, m = 1; len >= 1; len >>= 1, m <<= 1)
#pragma unroll
    for (int x = 0; x < n; ++x) {
      if ((x / len) & 1) continue;
      const int grp = x / (2 * len);
      const double t = fp_mulmod(a[x + len], T.psi_d[m + grp], T.qd, T.qinv);
      const double u = a[x];
      a[x] = __dadd_rn(u, t);
      a[x + len] = __dadd_rn(u, -t);
    }
  double* g = out + seg * n;
#pragma unroll
  for (int i = 0; i < n; ++i) g[i] = a[i];
}

// The double-precision kernels serve primes below 2^44 (exact products, ntt_fp.cuh).
static bool fp_ok(const NttTable& t0, const NttTable& t1) { return t0.q < (1ull << 44) && t1.q < (1ull << 44); }

// n = 2 and 4 on 8-bit digits: one thread per segment.
template <int LOGN>
__global__ void k_ntt_tiny_i8(const int8_t* __restrict__ din, u64* __restrict__ out, int nl, long segments,
                              NttTable t0, NttTable t1) {
  constexpr int n = 1 << LOGN;
  long seg = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (seg >= segments) return;
  const NttTable& T = (nl == 2 && (seg & 1)) ? t1 : t0;
  const u64 q = T.q;
  u64 a[n];
  const int8_t* gi = din + (seg / nl) * n;
#pragma unroll
  for (int i = 0; i < n; ++i) a[i] = gi[i] >= 0 ? (u64)gi[i] : q - (u64)(-gi[i]);
#pragma unroll
  for (int len = n / 2, m = 1; len >= 1; len >>= 1, m <<= 1)
#pragma unroll
    for (int x = 0; x < n; ++x) {
      if ((x / len) & 1) continue;
      const int grp = x / (2 * len);
      const u64 t = mul_shoup(a[x + len], T.psi[m + grp], T.psi_sh[m + grp], q);
      const u64 u = a[x];
      a[x] = addmod(u, t, q);
      a[x + len] = submod(u, t, q);
    }
  u64* g = out + seg * n;
#pragma unroll
  for (int i = 0; i < n; ++i) g[i] = a[i];
}

// n = 2 and 4: one thread per segment, all in registers.
template <int LOGN, bool INV>
__global__ void k_ntt_tiny(u64* __restrict__ data, int nl, long segments, NttTable t0, NttTable t1) {
  constexpr int n = 1 << LOGN;
  long seg = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (seg >= segments) return;
  const NttTable& T = (nl == 2 && (seg & 1)) ? t1 : t0;
  const u64 q = T.q;
  u64 a[n];
  u64* g = data + seg * n;
#pragma unroll
  for (int i = 0; i < n; ++i) a[i] = g[i];
  if (!INV) {
#pragma unroll
    for (int len = n / 2, m = 1; len >= 1; len >>= 1, m <<= 1)
#pragma unroll
      for (int x = 0; x < n; ++x) {
        if ((x / len) & 1) continue;
        const int grp = x / (2 * len);
        const u64 t = mul_shoup(a[x + len], T.psi[m + grp], T.psi_sh[m + grp], q);
        const u64 u = a[x];
        a[x] = addmod(u, t, q);
        a[x + len] = submod(u, t, q);
      }
  } else {
#pragma unroll
    for (int len = 1, m = n / 2; len < n; len <<= 1, m >>= 1)
#pragma unroll
      for (int x = 0; x < n; ++x) {
        if ((x / len) & 1) continue;
        const int grp = x / (2 * len);
        const u64 u = a[x], c = a[x + len];
        a[x] = addmod(u, c, q);
        a[x + len] = mul_shoup(submod(u, c, q), T.ipsi[m + grp], T.ipsi_sh[m + grp], q);
      }
#pragma unroll
    for (int i = 0; i < n; ++i) a[i] = mul_shoup(a[i], T.ninv[LOGN], T.ninv_sh[LOGN], q);
  }
#pragma unroll
  for (int i = 0; i < n; ++i) g[i] = a[i];
}

template <bool INV, bool LAZY = false>
static void launch(u64* data, int n, int nl, long segments, const NttTable& t0, const NttTable& t1,
                   cudaStream_t st) {
  if (segments <= 0) return;
  int logn = __builtin_ctz((unsigned)n);
  if (n < 2 || (n & (n - 1)) || logn > 12) throw CudaError(100, "ntt: degree must be a power of two in [2, 4096]");
  if (logn <= 2) {
    unsigned blocks = (unsigned)((segments + 127) / 128);
    if (logn == 1) k_ntt_tiny<1, INV><<<blocks, 128, 0, st>>>(data, nl, segments, t0, t1);
    else k_ntt_tiny<2, INV><<<blocks, 128, 0, st>>>(data, nl, segments, t0, t1);
    VIA_LAUNCHED();
    return;
  }
  const int cta = std::max(NTT_THREADS, n / 8);
  long spc = cta / (n / 8);
  unsigned blocks = (unsigned)((segments + spc - 1) / spc);
  const bool fp = fp_ok(t0, t1);
  switch (logn) {
#define VIA_NTT_CASE(LG)                                                              \
  case LG:                                                                           \
    if (fp)                                                                          \
      k_ntt_fp<LG, INV, LAZY><<<blocks, cta, 0, st>>>(data, nl, segments, t0, t1);   \
    else                                                                             \
      k_ntt_reg<LG, INV, LAZY><<<blocks, cta, 0, st>>>(data, nl, segments, t0, t1);  \
    break;
    VIA_NTT_CASE(3)
    VIA_NTT_CASE(4)
    VIA_NTT_CASE(5)
    VIA_NTT_CASE(6)
    VIA_NTT_CASE(7)
    VIA_NTT_CASE(8)
    VIA_NTT_CASE(9)
    VIA_NTT_CASE(10)
    VIA_NTT_CASE(11)
    VIA_NTT_CASE(12)
#undef VIA_NTT_CASE
  }
  VIA_LAUNCHED();
}

void ntt_forward(u64* data, int n, int nl, long segments, const NttTable& t0, const NttTable& t1, cudaStream_t st) {
  launch<false>(data, n, nl, segments, t0, t1, st);
}
void ntt_inverse(u64* data, int n, int nl, long segments, const NttTable& t0, const NttTable& t1, cudaStream_t st) {
  launch<true>(data, n, nl, segments, t0, t1, st);
}
void ntt_forward_lazy(u64* data, int n, int nl, long segments, const NttTable& t0, const NttTable& t1,
                      cudaStream_t st) {
  launch<false, true>(data, n, nl, segments, t0, t1, st);
}

void ntt_forward_i8_lazy(const int8_t* din, u64* out, int n, int nl, long segments, const NttTable& t0,
                         const NttTable& t1, cudaStream_t st) {
  if (segments <= 0) return;
  const int logn = __builtin_ctz((unsigned)n);
  if (n < 2 || (n & (n - 1)) || logn > 12) throw CudaError(100, "ntt: degree must be a power of two in [2, 4096]");
  if (logn <= 2) {
    const unsigned blocks = (unsigned)((segments + 127) / 128);
    if (logn == 1) k_ntt_tiny_i8<1><<<blocks, 128, 0, st>>>(din, out, nl, segments, t0, t1);
    else k_ntt_tiny_i8<2><<<blocks, 128, 0, st>>>(din, out, nl, segments, t0, t1);
    VIA_LAUNCHED();
    return;
  }
  const int cta = std::max(NTT_THREADS, n / 8);
  const long spc = cta / (n / 8);
  const unsigned blocks = (unsigned)((segments + spc - 1) / spc);
  const bool fp = fp_ok(t0, t1);
  switch (logn) {
#define VIA_NTT_I8_CASE(LG)                                                            \
  case LG:                                                                             \
    if (fp)                                                                            \
      k_ntt_fp_i8<LG><<<blocks, cta, 0, st>>>(din, out, nl, segments, t0, t1);         \
    else                                                                               \
      k_ntt_reg_i8<LG><<<blocks, cta, 0, st>>>(din, out, nl, segments, t0, t1);        \
    break;
    VIA_NTT_I8_CASE(3)
    VIA_NTT_I8_CASE(4)
    VIA_NTT_I8_CASE(5)
    VIA_NTT_I8_CASE(6)
    VIA_NTT_I8_CASE(7)
    VIA_NTT_I8_CASE(8)
    VIA_NTT_I8_CASE(9)
    VIA_NTT_I8_CASE(10)
    VIA_NTT_I8_CASE(11)
    VIA_NTT_I8_CASE(12)
#undef VIA_NTT_I8_CASE
  }
  VIA_LAUNCHED();
}

void ntt_forward_i8_fp(const int8_t* din, double* out, int n, int nl, long segments, const NttTable& t0,
                       const NttTable& t1, cudaStream_t st) {
  if (segments <= 0) return;
  const int logn = __builtin_ctz((unsigned)n);
  if (n < 2 || (n & (n - 1)) || logn > 12) throw CudaError(100, "ntt: degree must be a power of two in [2, 4096]");
  if (!fp_ok(t0, t1)) throw CudaError(100, "ntt: double-precision outputs need primes below 2^44");
  u64* o = reinterpret_cast<u64*>(out);
  if (logn <= 2) {
    const unsigned blocks = (unsigned)((segments + 127) / 128);
    if (logn == 1) k_ntt_tiny_i8_fp<1><<<blocks, 128, 0, st>>>(din, out, nl, segments, t0, t1);
    else k_ntt_tiny_i8_fp<2><<<blocks, 128, 0, st>>>(din, out, nl, segments, t0, t1);
    VIA_LAUNCHED();
    return;
  }
  const int cta = std::max(NTT_THREADS, n / 8);
  const long spc = cta / (n / 8);
  const unsigned blocks = (unsigned)((segments + spc - 1) / spc);
  switch (logn) {
#define VIA_NTT_I8D_CASE(LG) \
  case LG: k_ntt_fp_i8<LG, true><<<blocks, cta, 0, st>>>(din, o, nl, segments, t0, t1); break;
    VIA_NTT_I8D_CASE(3)
    VIA_NTT_I8D_CASE(4)
    VIA_NTT_I8D_CASE(5)
    VIA_NTT_I8D_CASE(6)
    VIA_NTT_I8D_CASE(7)
    VIA_NTT_I8D_CASE(8)
    VIA_NTT_I8D_CASE(9)
    VIA_NTT_I8D_CASE(10)
    VIA_NTT_I8D_CASE(11)
    VIA_NTT_I8D_CASE(12)
#undef VIA_NTT_I8D_CASE
  }
  VIA_LAUNCHED();
}

bool ntt_fp_ok(const NttTable& t0, const NttTable& t1) { return fp_ok(t0, t1); }

}  // namespace via
