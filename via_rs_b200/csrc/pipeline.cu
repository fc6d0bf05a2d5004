// The VIA-C answer pipeline on the device (crates/via-server/src/answer.rs:83-354):
//
//   1 QueryDecomp   LWE -> RLWE cascade (prim/conversion/cascade.rs) + RLWE -> RGSW
//   2 DMux tree     trivial RLWE(delta) -> I RLWEs at q1      (prim/gates/mux.rs:222)
//   3 ModSwitch     q1 -> q2                                   (prim/switching/mod_switch.rs:57)
//   4 FirstDim      I x J database scan                        (srv/first_dim.rs:94)
//   5 CMux tree     J -> 1 at q2                               (prim/gates/mux.rs:167)
//   6 CRot          slot extraction                            (prim/gates/rotate.rs:128)
//   7 RespComp      q2 -> q3, ring switch n1 -> n2, body -> q4 (srv/resp_comp.rs:46)
//
// Every gadget product is: exact decomposition into balanced digits (kernel
// k_decompose) -> forward NTT of the digit polys -> one pointwise
// multiply-accumulate against the eval-form key (k_mac) -> inverse NTT. Linear
// steps between products are done in whichever domain saves transforms; since
// the NTT is exact, the coefficient-form results equal the reference's.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "first_dim.cuh"
#include "gadget.cuh"
#include "ntt_fp.cuh"
#include "server.cuh"

namespace via {

// Grid size below which k_cascade_mac splits its output masks over more blocks.
constexpr long CASCADE_SPLIT_BLOCKS = 4 * 148;

// in: npolys polys [p][nl][n_in]; out: digit polys [p][L][nl][n_out] in sample
// order (slot s = L-1-k holds digit k). n_out = n_in * stride: the input is
// first embedded at slot 0 (reshape.rs:58), so other positions get digit 0.
__global__ void k_decompose(const u64* __restrict__ in, int n_in, int stride, long npolys, DevRing R, Gadget g,
                            u64* __restrict__ out) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= npolys * n_in) return;
  long p = gid / n_in;
  int i = (int)(gid % n_in);
  const int nl = R.nl;
  const u64* src = in + p * nl * n_in;
  u64 a0 = src[i], a1 = nl == 2 ? src[n_in + i] : 0;
  const int n_out = n_in * stride;
  const long step = (long)nl * n_out;
  // Digit k goes to sample slot L - 1 - k.
  u64* o = out + p * (long)g.L * step + (long)(g.L - 1) * step + (long)i * stride;
  for_each_digit(gadget_scaled(a0, a1, R, g), g, [&](int, i64 d) {
    for (int l = 0; l < nl; ++l) {
      u64* ol = o + (long)l * n_out;
      ol[0] = lift_i64(d, R.m[l]);
      for (int z = 1; z < stride; ++z) ol[z] = 0;
    }
    o -= step;
  });
}

// The same digits as signed bytes for gadgets with B <= 255 (|digit| <= 127),
// limb-free: out [p][L][n_in] in sample order; the 8-bit transforms lift them
// per limb. A sixteenth of the bytes of the u64 digits of a two-limb ring.
__global__ void k_decompose_i8(const u64* __restrict__ in, int n_in, long npolys, DevRing R, Gadget g,
                               int8_t* __restrict__ out) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= npolys * n_in) return;
  const long p = gid / n_in;
  const int i = (int)(gid % n_in);
  const int nl = R.nl;
  const u64* src = in + p * nl * n_in;
  const u64 a0 = src[i], a1 = nl == 2 ? src[n_in + i] : 0;
  int8_t* o = out + p * (long)g.L * n_in + (long)(g.L - 1) * n_in + i;
  for_each_digit(gadget_scaled(a0, a1, R, g), g, [&](int, i64 d) {
    *o = (int8_t)d;
    o -= n_in;
  });
}

// Which eval-form key samples output o multiplies: K_o = base + ((o / div) % mod) * stride.
// stride = 0 means "consecutive keys" (T*2*nl*n residues apart, T = samples per key).
struct KeySel {
  const u64* base;
  long div, mod, stride;
};
static inline KeySel keys_shared(const u64* base) { return KeySel{base, 1, 1, 0}; }
static inline KeySel keys_cyclic(const u64* base, long mod) { return KeySel{base, 1, mod, 0}; }

// ---------------------------------------------------------------------------
// Multiply-accumulate against eval-form keys.
//   out[o].{mask,body} = sum_{s<T} D[o*T + s] (*) K_o[s].{mask,body}
// K_o selected by a KeySel (T samples per key).
// ---------------------------------------------------------------------------
__global__ void k_mac_ntt(const u64* __restrict__ D, KeySel ks, u64* __restrict__ out, int T, int n, int nl, long nout,
                          DevRing R) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long per = (long)nl * n;
  if (gid >= nout * per) return;
  long o = gid / per;
  int rem = (int)(gid % per);
  int l = rem / n;
  const u64* Ko = ks.base + ((o / ks.div) % ks.mod) * (ks.stride ? ks.stride : (long)T * 2 * per);
  const u64* Do = D + o * (long)T * per;
  Acc128 am{0, 0}, ab{0, 0};
#pragma unroll 6
  for (int s = 0; s < T; ++s) {
    u64 dv = Do[s * per + rem];
    mac128(am, dv, Ko[(2 * s) * per + rem]);
    mac128(ab, dv, Ko[(2 * s + 1) * per + rem]);
  }
  const DevMod& m = R.m[l];
  out[(2 * o) * per + rem] = reduce128(am.hi, am.lo, m);
  out[(2 * o + 1) * per + rem] = reduce128(ab.hi, ab.lo, m);
}

// Schoolbook (non-NTT ring) variant: negacyclic products, exact.
__global__ void k_mac_schoolbook(const u64* __restrict__ D, KeySel ks, u64* __restrict__ out, int T, int n, int nl,
                                 long nout, DevRing R) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long per = (long)nl * n;
  if (gid >= nout * per) return;
  long o = gid / per;
  int rem = (int)(gid % per);
  int l = rem / n, t = rem % n;
  const u64* Ko = ks.base + ((o / ks.div) % ks.mod) * (ks.stride ? ks.stride : (long)T * 2 * per);
  const u64* Do = D + o * (long)T * per;
  const DevMod& m = R.m[l];
  const bool pow2 = m.log2q >= 0;
  u64 wm = 0, wb = 0;
  Acc128 pm{0, 0}, nm{0, 0}, pb{0, 0}, nb{0, 0};
  for (int s = 0; s < T; ++s) {
    const u64* dp = Do + s * per + (long)l * n;
    const u64* km = Ko + (2 * s) * per + (long)l * n;
    const u64* kb = Ko + (2 * s + 1) * per + (long)l * n;
    for (int j = 0; j < n; ++j) {
      u64 dv = dp[j];
      if (dv == 0) continue;
      int k = t - j;
      bool ng = k < 0;
      if (ng) k += n;
      if (pow2) {
        u64 a = dv * km[k], b = dv * kb[k];
        wm += ng ? (u64)0 - a : a;
        wb += ng ? (u64)0 - b : b;
      } else if (ng) {
        mac128(nm, dv, km[k]);
        mac128(nb, dv, kb[k]);
      } else {
        mac128(pm, dv, km[k]);
        mac128(pb, dv, kb[k]);
      }
    }
  }
  u64 rm, rb;
  if (pow2) {
    rm = wm & (m.q - 1);
    rb = wb & (m.q - 1);
  } else {
    rm = submod(reduce128(pm.hi, pm.lo, m), reduce128(nm.hi, nm.lo, m), m.q);
    rb = submod(reduce128(pb.hi, pb.lo, m), reduce128(nb.hi, nb.lo, m), m.q);
  }
  out[(2 * o) * per + rem] = rm;
  out[(2 * o + 1) * per + rem] = rb;
}

// ---------------------------------------------------------------------------
// Elementwise kernels. All buffers are [poly][limb][n].
// ---------------------------------------------------------------------------
// out[j] = a[j*sa] + sign * b[j*sb] for RLWEs (2 polys each); sign in {+1,-1}.
__global__ void k_rlwe_addsub(u64* out, const u64* a, long sa, const u64* b, long sb, int sign, long count, int n,
                              int nl, DevRing R) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long per = 2L * nl * n;
  if (gid >= count * per) return;
  long j = gid / per;
  int rem = (int)(gid % per);
  int l = (rem / n) % nl;
  u64 q = R.m[l].q;
  u64 x = a[j * sa * per + rem], y = b[j * sb * per + rem];
  out[j * per + rem] = sign > 0 ? addmod(x, y, q) : submod(x, y, q);
}

// The trivial RLWE (0, delta) at q1 (answer.rs:181-191): zero mask, body = delta * X^0.
// `count` trivial RLWEs (0, d) with d the constant (d0, d1) in RNS form.
__global__ void k_set_trivial(u64* ct, long count, int n, int nl, u64 d0, u64 d1) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= count * 2 * nl * n) return;
  const long r = gid % (2L * nl * n);
  const int poly = (int)(r / (nl * n)), rem = (int)(r % (nl * n));
  const int l = rem / n, i = rem % n;
  ct[gid] = (poly == 1 && i == 0) ? (l == 0 ? d0 : d1) : 0;
}

// DMux combine (mux.rs:129-137, 222-251): out[2j] = in[j] - ext[j], out[2j+1] = ext[j].
__global__ void k_dmux_combine(u64* out, const u64* in, const u64* ext, long count, int n, int nl, DevRing R) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long per = 2L * nl * n;
  if (gid >= count * per) return;
  long j = gid / per;
  int rem = (int)(gid % per);
  int l = (rem / n) % nl;
  u64 q = R.m[l].q;
  u64 e = ext[j * per + rem];
  out[(2 * j) * per + rem] = submod(in[j * per + rem], e, q);
  out[(2 * j + 1) * per + rem] = e;
}

// One DMux tree level in a single kernel (mux.rs:129-137, 222-251; the external
// product rgsw.rs:108-121 with the coefficient-form gadget product,
// rlev.rs:193-222), in double precision (ntt_fp.cuh). CTA (o, l) computes limb l
// of ext[o] = bit (x) in[o] and writes out[2o] = in[o] - ext, out[2o+1] = ext:
// the gadget digits (L = 2) of the mask and body coefficients (both limbs read,
// one CRT scaling per coefficient, digits kept in shared memory), forward
// transforms of the four digit polynomials at prime l, products with the RGSW
// samples (each within 0.5625 q; digit k of input half h with sample
// h L + L - 1 - k), and inverse transforms of the two sums (below 2.25 q).
// Buffers: [ct][2][nl][n], RGSW [2L][2][nl][n] eval at q1; nl = 2 primes below 2^44.
template <int LOGN>
__global__ void __launch_bounds__((1 << LOGN) / 8, 2) k_dmux_fp(u64* __restrict__ out, const u64* __restrict__ in,
                                                                  KeySel ks, DevRing R, Gadget g) {
  constexpr int n = 1 << LOGN;
  constexpr int L = 2;
  constexpr int nl = 2;
  using Fw0 = NttPhase<LOGN, false, 0>;
  using FwL = NttPhase<LOGN, false, (LOGN + 2) / 3 - 1>;
  using In0 = NttPhase<LOGN, true, 0>;
  using InL = NttPhase<LOGN, true, (LOGN + 2) / 3 - 1>;
  static_assert(In0::STRIDE == 1 && In0::R == 3 && FwL::STRIDE == 1, "contiguous end layouts");
  __shared__ double ssm[n];
  __shared__ int dgs[L][n];  // one half's digits; each thread reads back only its own slots
  const int tid = threadIdx.x;
  const long o = blockIdx.x;
  const int l = blockIdx.y;
  const NttTable& T = R.t[l];
  const double q = T.qd, qinv = T.qinv;
  const u64* ct = in + o * 2 * nl * n;
  const u64* K = ks.base + ((o / ks.div) % ks.mod) * ks.stride;
  double am[8], ab[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) am[v] = ab[v] = 0.0;
  for (int h = 0; h < 2; ++h) {  // 0: mask digits (neg_s_m rows), 1: body digits (m rows)
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const int x = Fw0::index(v, tid);
      const u64 a0 = ct[(long)h * nl * n + x], a1 = ct[(long)h * nl * n + n + x];
      for_each_digit(gadget_scaled(a0, a1, R, g), g, [&](int k, i64 d) { dgs[k][x] = (int)d; });
    }
#pragma unroll 1
    for (int k = 0; k < L; ++k) {
      double e[8];
#pragma unroll
      for (int v = 0; v < 8; ++v) e[v] = (double)dgs[k][Fw0::index(v, tid)];
      ntt_forward_fp<LOGN>(e, tid, T, ssm);
      const int smp = h * L + L - 1 - k;
      const ulonglong2* Km = reinterpret_cast<const ulonglong2*>(K + ((long)(2 * smp) * nl + l) * n + 8 * tid);
      const ulonglong2* Kb = reinterpret_cast<const ulonglong2*>(K + ((long)(2 * smp + 1) * nl + l) * n + 8 * tid);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const ulonglong2 km = __ldg(Km + c), kb = __ldg(Kb + c);
        am[2 * c] = __dadd_rn(am[2 * c], fp_mulmod(e[2 * c], __ull2double_rn(km.x), q, qinv));
        am[2 * c + 1] = __dadd_rn(am[2 * c + 1], fp_mulmod(e[2 * c + 1], __ull2double_rn(km.y), q, qinv));
        ab[2 * c] = __dadd_rn(ab[2 * c], fp_mulmod(e[2 * c], __ull2double_rn(kb.x), q, qinv));
        ab[2 * c + 1] = __dadd_rn(ab[2 * c + 1], fp_mulmod(e[2 * c + 1], __ull2double_rn(kb.y), q, qinv));
      }
    }
  }
  const u64 qi = R.m[l].q;
  u64* o0 = out + (2 * o) * 2 * nl * n;
  u64* o1 = o0 + 2 * nl * n;
  ntt_inverse_fp<LOGN, 0, true>(am, tid, T, ssm);
#pragma unroll
  for (int v = 0; v < 8; ++v) {  // ext mask
    const long at = (long)l * n + InL::index(v, tid);
    const u64 ext = __double2ull_rn(fp_canonical(am[v], q, qinv));
    o0[at] = submod(ct[at], ext, qi);
    o1[at] = ext;
  }
  __syncthreads();  // the body's transform reuses the exchange area
  ntt_inverse_fp<LOGN, 0, true>(ab, tid, T, ssm);
#pragma unroll
  for (int v = 0; v < 8; ++v) {  // ext body
    const long at = (long)(nl + l) * n + InL::index(v, tid);
    const u64 ext = __double2ull_rn(fp_canonical(ab[v], q, qinv));
    o0[at] = submod(ct[at], ext, qi);
    o1[at] = ext;
  }
}

// Inverse transforms of RLWEs ext ([count][2][nl][n], eval form, canonical) in
// double precision (ntt_fp.cuh), one CTA per polynomial, with the consumer's
// elementwise step folded into the stores (coefficient form, canonical):
//   INTT_STORE: out[j] = ext[j]
//   INTT_DMUX:  out[2j] = base[j] - ext[j], out[2j+1] = ext[j]  (a DMux level)
//   INTT_ADD:   out[j] = base[j] + ext[j]                       (a CRot step)
enum { INTT_STORE = 0, INTT_DMUX = 1, INTT_ADD = 2 };
template <int LOGN, int MODE>
__global__ void __launch_bounds__((1 << LOGN) / 8) k_intt_fp_epi(const u64* __restrict__ ext, const u64* base,
                                                                 u64* out, DevRing R) {
  constexpr int n = 1 << LOGN;
  using In0 = NttPhase<LOGN, true, 0>;
  using InL = NttPhase<LOGN, true, (LOGN + 2) / 3 - 1>;
  static_assert(In0::STRIDE == 1 && In0::R == 3, "contiguous first inverse layout");
  __shared__ double ssm[n];
  const int tid = threadIdx.x;
  const int nl = R.nl;
  const long seg = blockIdx.x;  // ((j * 2) + part) * nl + limb
  const int l = (int)(seg % nl);
  const NttTable& T = R.t[l];
  const double q = T.qd, qinv = T.qinv;
  double e[8];
  const ulonglong2* src = reinterpret_cast<const ulonglong2*>(ext + seg * n + 8 * tid);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const ulonglong2 x = src[c];
    e[2 * c] = __ull2double_rn(x.x);
    e[2 * c + 1] = __ull2double_rn(x.y);
  }
  ntt_inverse_fp<LOGN, 0, true>(e, tid, T, ssm);
  const u64 qi = R.m[l].q;
  const long per = 2L * nl * n, j = seg / (2 * nl), at0 = (seg % (2 * nl)) * n;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    const int x = InL::index(v, tid);
    const u64 val = __double2ull_rn(fp_canonical(e[v], q, qinv));
    if constexpr (MODE == INTT_STORE) {
      out[seg * n + x] = val;
    } else if constexpr (MODE == INTT_DMUX) {
      out[(2 * j) * per + at0 + x] = submod(base[j * per + at0 + x], val, qi);
      out[(2 * j + 1) * per + at0 + x] = val;
    } else {
      out[seg * n + x] = addmod(base[seg * n + x], val, qi);
    }
  }
}

// Runs k_intt_fp_epi for `count` RLWEs; false (nothing launched) when the ring
// has no double-precision transform of this degree.
template <int MODE>
static bool intt_epi(const DevRing& R, const u64* ext, const u64* base, u64* out, long count, cudaStream_t st) {
  if (!R.ntt || !ntt_fp_ok(R.t[0], R.t[R.nl - 1])) return false;
  const unsigned grid = (unsigned)(count * 2 * R.nl);
  switch (R.n) {
    case 4096: k_intt_fp_epi<12, MODE><<<grid, 512, 0, st>>>(ext, base, out, R); break;
    case 2048: k_intt_fp_epi<11, MODE><<<grid, 256, 0, st>>>(ext, base, out, R); break;
    case 1024: k_intt_fp_epi<10, MODE><<<grid, 128, 0, st>>>(ext, base, out, R); break;
    case 512: k_intt_fp_epi<9, MODE><<<grid, 64, 0, st>>>(ext, base, out, R); break;
    default: return false;
  }
  VIA_LAUNCHED();
  return true;
}

// Rings whose inverse transforms k_intt_fp_epi serves.
static bool R_fp_small(const DevRing& R) {
  return R.ntt && ntt_fp_ok(R.t[0], R.t[R.nl - 1]) && (R.n == 512 || R.n == 1024 || R.n == 2048 || R.n == 4096);
}

static bool dmux_fp_ok(const DevRing& R, const Gadget& g) {
  return R.ntt && R.nl == 2 && g.L == 2 && ntt_fp_ok(R.t[0], R.t[1]) && R.n == 2048;
}

// Modulus switch (prim/switching/kernels/mod_switch.rs:59-61):
// c' = floor((c * q_dst + floor(q_src/2)) / q_src) mod q_dst, c the canonical value.
__global__ void k_mod_switch(const u64* __restrict__ in, DevRing S, u64* __restrict__ out, DevMod dst, long ncoef,
                             int n, double dQs) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= ncoef) return;
  long p = gid / n;
  int i = (int)(gid % n);
  u128 v = S.nl == 2 ? crt2(in[(p * 2) * n + i], in[(p * 2 + 1) * n + i], S) : (u128)in[p * n + i];
  u128 Qs = S.Q();
  u128 num = v * dst.q + (Qs >> 1);
  u128 r;
  if (S.nl == 1 && S.m[0].log2q >= 0)
    r = num >> S.m[0].log2q;
  else
    r = div_exact(num, Qs, dQs);
  u64 rr = (u64)r;
  out[p * n + i] = rr >= dst.q ? rr - dst.q : rr;
}

// ---------------------------------------------------------------------------
// Cascade (prim/conversion/cascade.rs + conv.rs:122-148) helpers.
// ---------------------------------------------------------------------------
// LWE [lwe][nl*(n1+1)] -> rank-n1 MLWE of degree 1: masks [lwe][idx][nl], body [lwe][nl].
__global__ void k_lwe_to_mlwe(const u64* __restrict__ q, int n1, int nl, long nlwe, u64* masks, u64* body) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long per = (long)nl * (n1 + 1);
  if (gid >= nlwe * per) return;
  long w = gid / per;
  int r = (int)(gid % per);
  if (r < nl * n1) {
    int l = r / n1, idx = r % n1;
    masks[(w * n1 + idx) * nl + l] = q[w * per + r];
  } else {
    int l = r - nl * n1;
    body[w * nl + l] = q[w * per + r];
  }
}

// Regroups a batch's query LWEs: every query's first lwe_a LWEs (its DMux
// bits), query by query, then the rest of every query. Element-wise copy.
__global__ void k_permute_lwes(const u64* __restrict__ q, long nq, long n_lwe, long lwe_a, long lwe_len,
                               u64* __restrict__ out) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nq * n_lwe * lwe_len) return;
  const long e = gid % lwe_len, lw = gid / lwe_len;
  const long qi = lw / n_lwe, j = lw % n_lwe;
  const long dst = j < lwe_a ? qi * lwe_a + j : nq * lwe_a + qi * (n_lwe - lwe_a) + (j - lwe_a);
  out[dst * lwe_len + e] = q[gid];
}

// After the step MAC: P [lwe][RANK_IN][2][nl][N] (eval). Produces
// masks_out[lwe][j] = -(P[j].mask + P[j+R].mask) for j < R and
// bsum[lwe] = sum_idx P[idx].body.
__global__ void k_cascade_reduce(const u64* __restrict__ P, int rank_in, int N, int nl, long nlwe, DevRing R,
                                 u64* __restrict__ masks_out, u64* __restrict__ bsum) {
  const int half = rank_in / 2;
  long per = (long)nl * N;
  long items = nlwe * (half + 1) * per;
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= items) return;
  long w = gid / ((half + 1) * per);
  long r = gid % ((half + 1) * per);
  int j = (int)(r / per);
  int rem = (int)(r % per);
  int l = rem / N;
  u64 q = R.m[l].q;
  const u64* Pw = P + w * rank_in * 2 * per;
  if (j < half) {
    u64 a = Pw[(2L * j) * per + rem], b = Pw[(2L * (j + half)) * per + rem];
    masks_out[(w * half + j) * per + rem] = negmod(addmod(a, b, q), q);
  } else {
    u64 acc = 0;
    for (int idx = 0; idx < rank_in; ++idx) acc = addmod(acc, Pw[(2L * idx + 1) * per + rem], q);
    bsum[w * per + rem] = acc;
  }
}

// One cascade step's key switches and rank reduction in a single pass
// (conv.rs:122-148): the digits D of the R input masks are transformed at the
// input degree n_in, where the eval form of embed_at(d, 0) (d(X^2) of degree
// 2 n_in) is d's own eval form with every slot repeated (slot t of the output
// degree reads slot t/2). For every output mask j < R/2 and slot t:
//   mask_out[j] = -(sum_s D[j][s] K_j[s].mask + D[j+R/2][s] K_{j+R/2}[s].mask)
//   bsum        =   sum_idx sum_s D[idx][s] K_idx[s].body
// D: [lwe][idx][L][nl][n_in]; keys: [idx][L][2][nl][n_out]; mask_out:
// [lwe][R/2][nl][n_out]. Block = TT slots x JJ output masks (TT * JJ = 256); the
// JJ lanes' body partials are summed in shared memory. Small batches give few
// blocks: the output masks j are then also split over JB blocks (blockIdx.x =
// slot block * JB + jb). Every block adds its body partial (canonical, so at
// most JB of them sum below 2^64) into this step's region of the zeroed
// accumulator bsk: bsk[(lwe nl + l) * bsk_stride + t]. The body itself is only
// needed after the last step (k_cascade_body_final).
__global__ void __launch_bounds__(256) k_cascade_mac(const u64* __restrict__ D, const u64* __restrict__ keys, int R,
                                                     int n_in, int L, int TT, int JB, DevRing Rg,
                                                     u64* __restrict__ mask_out, u64* __restrict__ bsk,
                                                     long bsk_stride) {
  __shared__ u64 part[256];
  const int nl = Rg.nl, n_out = 2 * n_in, half = R / 2;
  const int JJ = 256 / TT;
  const int jb = blockIdx.x % JB;
  const int tl = threadIdx.x % TT, jl = threadIdx.x / TT;
  const int t = (blockIdx.x / JB) * TT + tl;
  const int l = blockIdx.y;
  const long lwe = blockIdx.z;
  const DevMod& m = Rg.m[l];
  const long dper = (long)nl * n_in, kper = (long)nl * n_out;
  const u64* Dw = D + lwe * R * L * dper + (long)l * n_in + (t >> 1);
  const u64* Kl = keys + (long)l * n_out + t;
  Acc128 ab{0, 0};
  for (int j = jl + jb * JJ; j < half; j += JJ * JB) {
    Acc128 am{0, 0};
    const u64* d0 = Dw + (long)j * L * dper;
    const u64* d1 = Dw + (long)(j + half) * L * dper;
    const u64* k0 = Kl + (long)j * L * 2 * kper;
    const u64* k1 = Kl + (long)(j + half) * L * 2 * kper;
#pragma unroll 3
    for (int s = 0; s < L; ++s) {
      const u64 a = d0[s * dper], b = d1[s * dper];
      mac128(am, a, k0[(2 * s) * kper]);
      mac128(am, b, k1[(2 * s) * kper]);
      mac128(ab, a, k0[(2 * s + 1) * kper]);
      mac128(ab, b, k1[(2 * s + 1) * kper]);
    }
    mask_out[((lwe * half + j) * nl + l) * n_out + t] = negmod(reduce128(am.hi, am.lo, m), m.q);
  }
  part[threadIdx.x] = reduce128(ab.hi, ab.lo, m);
  __syncthreads();
  if (jl == 0) {
    u64 acc = part[tl];
    for (int x = 1; x < JJ; ++x) acc = addmod(acc, part[x * TT + tl], m.q);
    if (JB == 1)
      bsk[(lwe * nl + l) * bsk_stride + t] = acc;
    else
      atomicAdd(reinterpret_cast<unsigned long long*>(bsk + (lwe * nl + l) * bsk_stride + t),
                (unsigned long long)acc);
  }
}

// k_cascade_mac in double precision (ntt_fp.cuh): D holds the digits' signed
// double transforms (ntt_forward_i8_fp, within 7 q of zero), keys the cascade
// key as exact doubles (below q). Every product is reduced to within 0.5625 q,
// so a mask's 2 L products stay below 1.125 L q; the body partial is brought
// back within q/2 after each output mask's 2 L products. Outputs as k_cascade_mac.
// Two CTAs per SM leave room for nine digits' loads in flight per thread.
// I8 (the first step, n_in = 1): the digits are read as the signed bytes of
// k_decompose_i8, [lwe][idx][L], whose transform at degree 1 is the digit itself.
template <bool I8>
__global__ void __launch_bounds__(256, 2) k_cascade_mac_fp(const double* __restrict__ D, const int8_t* __restrict__ D8,
                                                        const double* __restrict__ keys, int R, int n_in, int L,
                                                        int TT, int JB, DevRing Rg, u64* __restrict__ mask_out,
                                                        u64* __restrict__ bsk, long bsk_stride) {
  __shared__ u64 part[256];
  const int nl = Rg.nl, n_out = 2 * n_in, half = R / 2;
  const int JJ = 256 / TT;
  const int jb = blockIdx.x % JB;
  const int tl = threadIdx.x % TT, jl = threadIdx.x / TT;
  const int t = (blockIdx.x / JB) * TT + tl;
  const int l = blockIdx.y;
  const long lwe = blockIdx.z;
  const DevMod& m = Rg.m[l];
  const double q = Rg.t[l].qd, qinv = Rg.t[l].qinv;
  const long dper = (long)nl * n_in, kper = (long)nl * n_out;
  const double* Dw = D + lwe * R * L * dper + (long)l * n_in + (t >> 1);
  const double* Kl = keys + (long)l * n_out + t;
  double ab = 0.0;
  for (int j = jl + jb * JJ; j < half; j += JJ * JB) {
    double am = 0.0;
    const double* d0 = Dw + (long)j * L * dper;
    const double* d1 = Dw + (long)(j + half) * L * dper;
    const double* k0 = Kl + (long)j * L * 2 * kper;
    const double* k1 = Kl + (long)(j + half) * L * 2 * kper;
    const int8_t* e0 = D8 + (lwe * R + j) * L;
    const int8_t* e1 = D8 + (lwe * R + j + half) * L;
#pragma unroll 9
    for (int s = 0; s < L; ++s) {
      const double a = I8 ? (double)e0[s] : d0[s * dper], b = I8 ? (double)e1[s] : d1[s * dper];
      am = __dadd_rn(am, __dadd_rn(fp_mulmod(a, k0[(2 * s) * kper], q, qinv), fp_mulmod(b, k1[(2 * s) * kper], q, qinv)));
      ab = __dadd_rn(ab, __dadd_rn(fp_mulmod(a, k0[(2 * s + 1) * kper], q, qinv),
                                   fp_mulmod(b, k1[(2 * s + 1) * kper], q, qinv)));
    }
    mask_out[((lwe * half + j) * nl + l) * n_out + t] = negmod(__double2ull_rn(fp_canonical(am, q, qinv)), m.q);
    ab = __fma_rn(-__dadd_rn(__fma_rn(ab, qinv, FP_ROUND), -FP_ROUND), q, ab);  // back within q/2
  }
  part[threadIdx.x] = __double2ull_rn(fp_canonical(ab, q, qinv));
  __syncthreads();
  if (jl == 0) {
    u64 acc = part[tl];
    for (int x = 1; x < JJ; ++x) acc = addmod(acc, part[x * TT + tl], m.q);
    if (JB == 1)
      bsk[(lwe * nl + l) * bsk_stride + t] = acc;
    else
      atomicAdd(reinterpret_cast<unsigned long long*>(bsk + (lwe * nl + l) * bsk_stride + t),
                (unsigned long long)acc);
  }
}

// The cascade's final body in the eval domain, [lwe][nl][n1] (n1 = 2^K). Step k
// (output degree 2^(k+1)) maps body to embed_at(body, 0) - bsum_k, and the eval
// form of embed_at repeats every slot, so
//   body[t] = b - sum_k bsum_k[t >> (K - 1 - k)]
// with b the LWE body (the degree-1 body, [lwe][nl]) and bsum_k the step's
// accumulated sums, bsk[(lwe nl + l) * 2 n1 + 2^(k+1) - 2 + slot].
__global__ void k_cascade_body_final(const u64* __restrict__ b0, const u64* __restrict__ bsk, int K, int nl,
                                     long nlwe, DevRing Rg, u64* __restrict__ body) {
  const int n1 = 1 << K;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nlwe * nl * n1) return;
  const long ll = gid / n1;  // lwe * nl + l
  const int t = (int)(gid % n1), l = (int)(ll % nl);
  const DevMod& m = Rg.m[l];
  const u64* sk = bsk + ll * 2 * n1;
  u64 acc = 0;
  for (int k = 0; k < K; ++k) acc = addmod(acc, reduce64(sk[(2 << k) - 2 + (t >> (K - 1 - k))], m), m.q);
  body[gid] = submod(b0[ll], acc, m.q);
}

// body_out[lwe] = embed_at(body_in[lwe], N_out, 0) - bsum[lwe] (coefficient form).
__global__ void k_cascade_body(const u64* __restrict__ body_in, const u64* __restrict__ bsum, int n_in, int nl,
                               long nlwe, DevRing R, u64* __restrict__ body_out) {
  const int n_out = 2 * n_in;
  long per = (long)nl * n_out;
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nlwe * per) return;
  long w = gid / per;
  int rem = (int)(gid % per);
  int l = rem / n_out, t = rem % n_out;
  u64 q = R.m[l].q;
  u64 e = (t & 1) ? 0 : body_in[(w * nl + l) * n_in + t / 2];
  body_out[w * per + rem] = submod(e, bsum[w * per + rem], q);
}

// Assemble cascade outputs into RLWEs [lwe][2][nl][n1].
__global__ void k_pack_rlwe(const u64* masks, const u64* body, long nlwe, int n1, int nl, u64* out) {
  long per = (long)nl * n1;
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nlwe * per) return;
  long w = gid / per;
  int rem = (int)(gid % per);
  out[(2 * w) * per + rem] = masks[w * per + rem];
  out[(2 * w + 1) * per + rem] = body[w * per + rem];
}

// rlwe_to_rgsw assembly (prim/gates/convert.rs:162-178): for bit b, level i:
// neg_s_m[i] = (rlwe_i.body + gp_i.mask, gp_i.body), m[i] = rlwe_i.
// rlwe: [bits*L][2][nl][n]; gp: same shape; rgsw: [bits][2L][2][nl][n].
__global__ void k_assemble_rgsw(const u64* rlwe, const u64* gp, int L, long bits, int n, int nl, DevRing R, u64* rgsw) {
  long per = (long)nl * n;
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= bits * L * 2 * per) return;
  long w = gid / (2 * per);  // rlwe index = bit*L + i
  int rem = (int)(gid % (2 * per));
  int mb = rem / per;
  int r2 = rem % per;
  int l = r2 / n;
  long b = w / L;
  int i = (int)(w % L);
  u64 q = R.m[l].q;
  u64* dst_nsm = rgsw + ((b * 2 * L + i) * 2 + mb) * per + r2;
  u64* dst_m = rgsw + ((b * 2 * L + L + i) * 2 + mb) * per + r2;
  u64 g = gp[(2 * w + mb) * per + r2];
  if (mb == 0)
    *dst_nsm = addmod(rlwe[(2 * w + 1) * per + r2], g, q);
  else
    *dst_nsm = g;
  *dst_m = rlwe[(2 * w + mb) * per + r2];
}

// CRot (rotate.rs:128-150, SlotExtract): rot = -(X^(n - 2^i) * ct); diff = rot - ct.
__global__ void k_crot_diff(const u64* ct, int n, int k, DevMod m, u64* diff) {
  int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= 2 * n) return;
  int p = gid / n, i = gid % n;
  // (X^k * a)[i] = a[i-k] (negated on wrap); rot = -(that).
  int src = i - k;
  bool wrap = src < 0;
  if (wrap) src += n;
  u64 v = ct[p * n + src];
  u64 xk = wrap ? negmod(v, m.q) : v;
  u64 rot = negmod(xk, m.q);
  diff[p * n + i] = submod(rot, ct[p * n + i], m.q);
}

// Ring switch inputs (prim/switching/ring_switch.rs:358-385): for j < d,
// mask_proj_j[t] = (X^j * mask)[d t]; body_proj_0[t] = body[d t].
__global__ void k_ring_switch_proj(const u64* ct, int n1, int n2, DevMod m, u64* mask_proj, u64* body_proj) {
  int d = n1 / n2;
  int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (d + 1) * n2) return;
  int j = gid / n2, t = gid % n2;
  if (j == d) {
    body_proj[t] = ct[n1 + d * t];
    return;
  }
  int src = d * t - j;
  bool wrap = src < 0;
  if (wrap) src += n1;
  u64 v = ct[src];
  mask_proj[j * n2 + t] = wrap ? negmod(v, m.q) : v;
}

// acc over j of gp_j (eval or coeff, summed as residues): out = -(sum mask), body_proj - sum body.
__global__ void k_ring_switch_sum(const u64* gp, int d, int n2, DevMod m, u64* acc) {
  int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= 2 * n2) return;
  int mb = gid / n2, t = gid % n2;
  u64 s = 0;
  for (int j = 0; j < d; ++j) s = addmod(s, gp[(2 * j + mb) * n2 + t], m.q);
  acc[mb * n2 + t] = s;
}

__global__ void k_ring_switch_finish(const u64* acc, const u64* body_proj, int n2, DevMod m3, DevMod m4, double dq3,
                                     u64* out_mask, u64* out_body) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n2) return;
  u64 q3 = m3.q;
  u64 mask = negmod(acc[t], q3);
  u64 body = submod(body_proj[t], acc[n2 + t], q3);
  out_mask[t] = mask;  // mask: q3 -> q3 is the identity rescale
  // body: q3 -> q4 (mod_switch_asym, prim/switching/mod_switch.rs:124-154).
  u128 num = (u128)body * m4.q + q3 / 2;
  u64 r = (u64)div_exact(num, (u128)q3, dq3);
  out_body[t] = r >= m4.q ? r - m4.q : r;
}

// ---------------------------------------------------------------------------
// Host-side orchestration.
// ---------------------------------------------------------------------------
static inline unsigned blocks(long items, int threads = 256) { return (unsigned)((items + threads - 1) / threads); }

struct Workspace {
  long nlwe = 0, nbits = 0;  // per query
  int bmax = 1;              // queries the buffers are sized for
  // Cascade.
  DevBuf c_masks_a, c_masks_b, c_body_a, c_body_b, c_digits, c_P, c_bsum, c_rlwe;
  DevBuf c_dig8;   // 8-bit cascade / conversion-key digits [lwe][n1 * L_CK] bytes (base <= 255)
  // RLWE -> RGSW.
  // RGSWs grouped by use: the DMux bits of every query ([q][nd]), then the
  // CMux and CRot bits ([q][nbits - nd]), each [2L][2][nl][n1] at q1.
  DevBuf g_digits, g_gp, rgsw_q1;
  DevBuf rgsw_q2;  // the same layout switched to q2: [2L][2][n1] per bit
  DevBuf q_perm;   // a batch's query LWEs in that grouped order (batches of two or more)
  // DMux.
  DevBuf dm_a, dm_b, dm_digits, dm_ext;
  // FirstDim / CMux.
  DevBuf sel, sel_bytes, fd_out, cm_diff, cm_digits, cm_ext, cm_b;
  // CRot / RespComp.
  DevBuf cr_ct, cr_diff, cr_digits, cr_ext, rs_ct3, rs_mproj, rs_bproj, rs_digits, rs_gp, rs_acc;
  Gadget g_ck, g_dmux, g_cmux, g_rsk;
  // Staging for the captured answer graphs: queries in, answers out.
  DevBuf q_in, a_mask, a_body;
  std::vector<std::pair<int, cudaGraphExec_t>> graphs;  // one per batch size
  std::vector<std::pair<int, unsigned long long>> graph_kernels;
  std::unique_ptr<struct RepackWs> repack;  // VIA-B buffers, made on the first batch answer
  cudaStream_t capture = nullptr;           // stream the answer graphs are captured on
  int graphs_gen = 0;                       // Server::plan_gen the graphs were captured under
  // A one-query answer expands its CMux / CRot bits on `side`, concurrently with
  // the DMux tree and the database scan on the answer's stream (fork / join).
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  ~Workspace() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    if (capture) cudaStreamDestroy(capture);
    if (side) cudaStreamDestroy(side);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
  }
};

void WorkspaceDeleter::operator()(Workspace* w) const { delete w; }
void workspace_destroy(Server& s) { s.ws.reset(); }
uint8_t* workspace_sel_bytes(Server& s) { return reinterpret_cast<uint8_t*>(s.ws->sel_bytes.p); }

void first_dim_queries(Server& s, const u64* sel_eval, u64* out_eval, int nq, uint8_t* scratch, cudaStream_t st) {
  const via_params& p = s.prm;
  if (s.tensor_fd()) {
    fd_scan(s.fd, sel_eval, out_eval, nq, scratch, st);
    return;
  }
  for (int q = 0; q < nq; ++q)
    first_dim_schoolbook(s.db->p, sel_eval + (size_t)q * p.num_rows * 2 * p.n1, out_eval + (size_t)q * p.num_cols * 2 * p.n1,
                         (int)p.num_rows, (int)p.num_cols, (int)p.n1, s.r2.m[0], st);
}

// Times every candidate scan tile for nq queries on the handle's workspace
// buffers (the workspace must hold batches of nq).
std::vector<FdTuneResult> workspace_measure_tiles(Server& s, Workspace& w, int nq, int reps) {
  if (w.bmax < nq) throw CudaError(100, "workspace smaller than the batch to tune");
  return fd_measure_tiles(s.fd, nq, w.sel.p, w.fd_out.p, reinterpret_cast<uint8_t*>(w.sel_bytes.p), s.stream, reps);
}

static bool cmux_fused_ok(const DevRing& R, const Gadget& g);

// Allocates a workspace for batches of up to bmax queries, or (count_only)
// returns the bytes it would take.
static size_t workspace_build(Server& s, int bmax, Workspace* w, bool count_only) {
  const via_params& p = s.prm;
  size_t bytes = 0;
  auto A = [&](DevBuf& b, long count) {
    bytes += (size_t)std::max(0L, count) * 8;
    if (!count_only) b.alloc((size_t)std::max(0L, count));
  };
  const long n1 = p.n1, n2 = p.n2, nl = s.r1.nl, L = p.l_query, Lck = p.l_ck, I = p.num_rows, J = p.num_cols;
  const long B = std::max(1, bmax);
  w->bmax = (int)B;
  w->nlwe = (long)query_lwes(p);
  w->nbits = w->nlwe / L;
  const long nlwe = w->nlwe * B;  // LWEs of a full batch
  A(w->c_masks_a, nlwe * n1 * nl);
  A(w->c_masks_b, nlwe * n1 * nl);
  A(w->c_body_a, nlwe * n1 * nl);
  A(w->c_body_b, nlwe * n1 * nl);
  // NTT rings transform the cascade digits at the input degree (half of the
  // embedded degree); the other rings use the embedded digits and the P buffer.
  A(w->c_digits, nlwe * (s.r1.ntt ? 1 : 2) * n1 * Lck * nl);
  A(w->c_P, s.r1.ntt ? 0 : nlwe * 2 * n1 * 2 * nl);
  A(w->c_bsum, 2 * nlwe * n1 * nl);
  A(w->c_dig8, p.ck_base <= 255 && s.r1.ntt ? (nlwe * n1 * Lck + 7) / 8 : 0);
  A(w->c_rlwe, nlwe * 2 * n1 * nl);
  A(w->g_digits, nlwe * Lck * nl * n1);
  A(w->g_gp, nlwe * 2 * nl * n1);
  A(w->rgsw_q1, B * w->nbits * 2 * L * 2 * nl * n1);
  A(w->rgsw_q2, B * w->nbits * 2 * L * 2 * n1);
  A(w->dm_a, B * I * 2 * nl * n1);
  A(w->dm_b, B * I * 2 * nl * n1);
  A(w->dm_digits, B * std::max(1L, I / 2) * 2 * L * nl * n1);
  A(w->dm_ext, B * std::max(1L, I / 2) * 2 * nl * n1);
  A(w->sel, B * I * 2 * n1);
  if (s.tensor_fd()) {
    size_t bytes = 0;  // the split selection grows with the batch; size it for every batch up to B
    for (int nq = 1; nq <= B; ++nq) bytes = std::max(bytes, fd_sel_bytes(s.fd, nq));
    A(w->sel_bytes, (bytes + 7) / 8);
  }
  A(w->fd_out, B * J * 2 * n1);
  const bool fused = cmux_fused_ok(s.r2, make_gadget(p.b_cmux, (int)p.l_query, s.r2));
  A(w->cm_diff, fused ? 0 : B * std::max(1L, J / 2) * 2 * n1);
  A(w->cm_digits, fused ? 0 : B * std::max(1L, J / 2) * 2 * L * n1);
  A(w->cm_ext, fused ? 0 : B * std::max(1L, J / 2) * 2 * n1);
  A(w->cm_b, B * std::max(1L, J / 2) * 2 * n1);
  A(w->cr_ct, B * 2 * n1);
  A(w->cr_diff, B * 2 * n1);
  A(w->cr_digits, B * 2 * L * n1);
  A(w->cr_ext, B * 2 * n1);
  A(w->rs_ct3, B * 2 * n1);
  long d = n1 / n2;
  A(w->rs_mproj, B * d * n2);
  A(w->rs_bproj, B * n2);
  A(w->rs_digits, B * d * p.l_rsk * n2);
  A(w->rs_gp, B * d * 2 * n2);
  A(w->rs_acc, B * 2 * n2);
  A(w->q_in, nlwe * lwe_len(p));
  A(w->q_perm, B > 1 ? nlwe * (long)lwe_len(p) : 0);
  A(w->a_mask, B * n2);
  A(w->a_body, B * n2);
  if (count_only) return bytes;
  w->g_ck = make_gadget(p.ck_base, (int)p.l_ck, s.r1);
  w->g_dmux = make_gadget(p.b_dmux, (int)p.l_query, s.r1);
  w->g_cmux = make_gadget(p.b_cmux, (int)p.l_query, s.r2);
  w->g_rsk = make_gadget(p.b_rsk, (int)p.l_rsk, s.r3);
  return bytes;
}

std::unique_ptr<Workspace, WorkspaceDeleter> workspace_make(Server& s, int bmax) {
  std::unique_ptr<Workspace, WorkspaceDeleter> w(new Workspace());
  workspace_build(s, bmax, w.get(), false);
  VIA_CUDA(cudaStreamCreateWithFlags(&w->capture, cudaStreamNonBlocking));
  VIA_CUDA(cudaStreamCreateWithFlags(&w->side, cudaStreamNonBlocking));
  VIA_CUDA(cudaEventCreateWithFlags(&w->ev_fork, cudaEventDisableTiming));
  VIA_CUDA(cudaEventCreateWithFlags(&w->ev_join, cudaEventDisableTiming));
  return w;
}

size_t workspace_bytes(Server& s, int bmax) {
  Workspace scratch;
  return workspace_build(s, bmax, &scratch, true);
}

void workspace_create(Server& s, int bmax) { s.ws = workspace_make(s, bmax); }


int workspace_batch(Server& s) { return s.ws ? s.ws->bmax : 0; }

static void to_eval(const DevRing& R, u64* data, int n, long segments, cudaStream_t st) {
  if (R.ntt) ntt_forward(data, n, R.nl, segments, R.t[0], R.t[1], st);
}
// Eval form of gadget digits: the lazy forward transform (outputs below
// (1 + 2 log2 n) q < 2^44 for q < 2^40, n <= 4096); their consumers add at most
// a few dozen products with key residues below q into 128-bit sums.
static void digits_to_eval(const DevRing& R, u64* data, int n, long segments, cudaStream_t st) {
  if (R.ntt) ntt_forward_lazy(data, n, R.nl, segments, R.t[0], R.t[1], st);
}
static void from_eval(const DevRing& R, u64* data, int n, long segments, cudaStream_t st) {
  if (R.ntt) ntt_inverse(data, n, R.nl, segments, R.t[0], R.t[1], st);
}

// Gadget products of `nout` outputs with T digit polys each (already in the eval
// domain) against keys: out eval [nout][2][nl][n].
static void mac(const DevRing& R, const u64* D, KeySel ks, u64* out, int T, int n, long nout, cudaStream_t st) {
  long items = nout * R.nl * n;
  if (R.ntt)
    k_mac_ntt<<<blocks(items), 256, 0, st>>>(D, ks, out, T, n, R.nl, nout, R);
  else
    k_mac_schoolbook<<<blocks(items), 256, 0, st>>>(D, ks, out, T, n, R.nl, nout, R);
  VIA_LAUNCHED();
}

static void decompose(const DevRing& R, const Gadget& g, const u64* in, int n_in, int stride, long npolys, u64* out,
                      cudaStream_t st) {
  k_decompose<<<blocks(npolys * n_in, 128), 128, 0, st>>>(in, n_in, stride, npolys, R, g, out);
  VIA_LAUNCHED();
}

// Gadget products of `nout` outputs, each summing G decomposed input polys
// against its eval-form key samples: decompose -> transform -> multiply-accumulate
// through the `digits` scratch ([nout][G][L][nl][n]).
static void gadget_product(const DevRing& R, const Gadget& g, const u64* in, int n, int stride, int G, long nout,
                           KeySel ks, u64* out, u64* digits, cudaStream_t st) {
  decompose(R, g, in, n / stride, stride, (long)G * nout, digits, st);
  digits_to_eval(R, digits, n, (long)G * nout * g.L * R.nl, st);
  mac(R, digits, ks, out, G * g.L, n, nout, st);
}

static double to_double(u128 x) { return (double)(u64)(x >> 64) * 18446744073709551616.0 + (double)(u64)x; }

static void mod_switch(const DevRing& S, const u64* in, const DevRing& D, u64* out, long npolys, int n, cudaStream_t st) {
  long nco = npolys * n;
  k_mod_switch<<<blocks(nco), 256, 0, st>>>(in, S, out, D.m[0], nco, n, to_double(S.Q()));
  VIA_LAUNCHED();
}

// Step 1: QueryDecomp (query_decomp.rs:39-95) of `nlwe` consecutive LWEs, the
// first being LWE lwe0 of the workspace (LWE-indexed buffers are used from that
// LWE's region on), forming the RGSWs of `nbits` query bits starting at bit
// bit0 -> rgsw_q1 [bit][2L][2][nl][n1] (coefficient form). Disjoint (lwe0,
// nlwe) ranges may run concurrently on different streams.
static void query_decomp_range(Server& s, Workspace& w, const u64* d_query, long lwe0, long nlwe, long bit0,
                               long nbits, cudaStream_t st) {
  const via_params& p = s.prm;
  const DevRing& R = s.r1;
  const int n1 = p.n1, nl = R.nl, L = p.l_ck;
  const long lwe_n = (long)n1 * nl;  // per-LWE region of the mask / body / bsum buffers
  const long rgsw1 = 2L * p.l_query * 2 * nl * n1;
  u64 *mi = w.c_masks_a.p + lwe0 * lwe_n, *mo = w.c_masks_b.p + lwe0 * lwe_n;
  u64 *bi = w.c_body_a.p + lwe0 * lwe_n, *bo = w.c_body_b.p + lwe0 * lwe_n;
  u64* digits = w.c_digits.p + lwe0 * (R.ntt ? 1 : 2) * n1 * L * nl;
  u64* cP = R.ntt ? nullptr : w.c_P.p + lwe0 * 2 * n1 * 2 * nl;
  u64* bsum = w.c_bsum.p + lwe0 * lwe_n;
  // Eval rings: every step's body sums, [lwe][nl][2 n1] (step regions of 2, 4, .. n1).
  u64* bsk = w.c_bsum.p + lwe0 * 2 * lwe_n;
  u64* rlwe = w.c_rlwe.p + lwe0 * 2 * lwe_n;
  // Bases up to 255: digits as bytes, lifted and transformed by the 8-bit NTT.
  int8_t* dig8 = w.c_dig8.p ? reinterpret_cast<int8_t*>(w.c_dig8.p) + lwe0 * (long)n1 * L : nullptr;
  k_lwe_to_mlwe<<<blocks(nlwe * nl * (n1 + 1)), 256, 0, st>>>(d_query + lwe0 * (long)lwe_len(p), n1, nl, nlwe, mi, bi);
  VIA_LAUNCHED();
  if (R.ntt) VIA_CUDA(cudaMemsetAsync(bsk, 0, (size_t)nlwe * 2 * lwe_n * 8, st));
  const u64 step_len = (u64)2 * n1 * L * 2 * nl;
  int k = 0;
  for (int n_in = 1; n_in < n1; n_in <<= 1, ++k) {
    const int n_out = 2 * n_in, rank_in = n1 / n_in;
    const long polys = nlwe * rank_in;
    if (R.ntt) {
      // Digits at the input degree; see k_cascade_mac for the repeated slots.
      const bool fp_mac = dig8 && s.cascade_eval_d.p;
      if (dig8 && (n_in > 1 || fp_mac)) {
        k_decompose_i8<<<blocks(polys * n_in, 128), 128, 0, st>>>(mi, n_in, polys, R, w.g_ck, dig8);
        VIA_LAUNCHED();
        if (n_in == 1)
          ;  // degree 1: the MAC reads the digits themselves
        else if (fp_mac)
          ntt_forward_i8_fp(dig8, reinterpret_cast<double*>(digits), n_in, nl, polys * L * nl, R.t[0], R.t[1], st);
        else
          ntt_forward_i8_lazy(dig8, digits, n_in, nl, polys * L * nl, R.t[0], R.t[1], st);
      } else {
        decompose(R, w.g_ck, mi, n_in, 1, polys, digits, st);
        if (n_in > 1) digits_to_eval(R, digits, n_in, polys * L * nl, st);
      }
      int jj = std::min(rank_in / 2, 8), tt = std::min(n_out, 256 / jj);
      // Split the output masks over JB blocks while the grid is below ~4 blocks
      // per SM and every block keeps at least one mask per thread row.
      const long base = (long)(n_out / tt) * nl * nlwe;
      const int iters = (rank_in / 2 + 256 / tt - 1) / (256 / tt);
      int JB = 1;
      while (JB * 2 <= iters && base * JB * 2 <= CASCADE_SPLIT_BLOCKS) JB *= 2;
      dim3 grid((unsigned)(n_out / tt * JB), (unsigned)nl, (unsigned)nlwe);
      u64* bsk_k = bsk + (n_out - 2);  // this step's region
      const double* kd = reinterpret_cast<const double*>(s.cascade_eval_d.p) + k * step_len;
      if (fp_mac && n_in == 1)
        k_cascade_mac_fp<true><<<grid, 256, 0, st>>>(nullptr, dig8, kd, rank_in, n_in, L, tt, JB, R, mo, bsk_k, 2L * n1);
      else if (fp_mac)
        k_cascade_mac_fp<false><<<grid, 256, 0, st>>>(reinterpret_cast<const double*>(digits), dig8, kd, rank_in, n_in,
                                                      L, tt, JB, R, mo, bsk_k, 2L * n1);
      else
        k_cascade_mac<<<grid, 256, 0, st>>>(digits, s.cascade_eval.p + k * step_len, rank_in, n_in, L, tt, JB, R, mo,
                                            bsk_k, 2L * n1);
      VIA_LAUNCHED();
      // The masks return to coefficient form for the next step's digits.
      from_eval(R, mo, n_out, nlwe * (rank_in / 2) * nl, st);
      std::swap(mi, mo);
      continue;
    } else {
      gadget_product(R, w.g_ck, mi, n_out, 2, 1, polys, keys_cyclic(s.cascade_eval.p + k * step_len, rank_in), cP,
                     digits, st);
      const long items = nlwe * (rank_in / 2 + 1) * nl * n_out;
      k_cascade_reduce<<<blocks(items), 256, 0, st>>>(cP, rank_in, n_out, nl, nlwe, R, mo, bsum);
      VIA_LAUNCHED();
      k_cascade_body<<<blocks(nlwe * nl * n_out), 256, 0, st>>>(bi, bsum, n_in, nl, nlwe, R, bo);
      VIA_LAUNCHED();
    }
    std::swap(mi, mo);
    std::swap(bi, bo);
  }
  if (R.ntt) {  // the cascade's body, from the LWE bodies in bi and every step's sums
    k_cascade_body_final<<<blocks(nlwe * nl * n1), 256, 0, st>>>(bi, bsk, k, nl, nlwe, R, bo);
    VIA_LAUNCHED();
    from_eval(R, bo, n1, nlwe * nl, st);
    std::swap(bi, bo);
  }
  k_pack_rlwe<<<blocks(nlwe * nl * n1), 256, 0, st>>>(mi, bi, nlwe, n1, nl, rlwe);
  VIA_LAUNCHED();
  // RLWE -> RGSW with the conversion key (prim/gates/convert.rs:162-178); the
  // final rank-1 masks are already contiguous [lwe][nl][n1] in `mi`.
  u64* gp = w.g_gp.p + lwe0 * 2 * lwe_n;
  u64* gdig = w.g_digits.p + lwe0 * L * lwe_n;
  if (dig8) {
    k_decompose_i8<<<blocks(nlwe * n1, 128), 128, 0, st>>>(mi, n1, nlwe, R, w.g_ck, dig8);
    VIA_LAUNCHED();
    ntt_forward_i8_lazy(dig8, gdig, n1, nl, nlwe * L * nl, R.t[0], R.t[1], st);
    mac(R, gdig, keys_shared(s.conv_eval.p), gp, L, n1, nlwe, st);
  } else {
    gadget_product(R, w.g_ck, mi, n1, 1, 1, nlwe, keys_shared(s.conv_eval.p), gp, gdig, st);
  }
  from_eval(R, gp, n1, nlwe * 2 * nl, st);
  k_assemble_rgsw<<<blocks(nlwe * 2 * nl * n1), 256, 0, st>>>(rlwe, gp, (int)p.l_query, nbits, n1, nl, R,
                                                               w.rgsw_q1.p + bit0 * rgsw1);
  VIA_LAUNCHED();
}


// ext[o] = bit_o (x) cts[o] for `count` RLWEs (coefficient form); result in the
// eval domain unless `to_coeff`. The RGSW of output o is selected by `rgsw`.
static void external_products(const DevRing& R, const Gadget& g, KeySel rgsw, const u64* cts, long count, u64* digits,
                              u64* ext, bool to_coeff, cudaStream_t st) {
  const int n = R.n;
  // Mask and body of every RLWE are the G = 2 decomposed inputs; their digits
  // pair with the neg_s_m and m samples of the RGSW respectively.
  gadget_product(R, g, cts, n, 1, 2, count, rgsw, ext, digits, st);
  if (to_coeff) from_eval(R, ext, n, 2 * count * R.nl, st);
}

// One CMux of a tree level per CTA (mux.rs:75-84, 167-198; rgsw.rs:108-121),
// single-limb ring of degree 2^LOGN with a small gadget (gadget_scaled_small),
// 2^LOGN / 8 threads holding 8 residues each:
//   diff = in[2o+1] - in[2o] (eval) -> inverse NTT -> balanced digits of the
//   mask and body -> forward NTT of each digit polynomial -> products with the
//   RGSW samples (mask digits with neg_s_m, body digits with m, digit k with
//   sample L-1-k) -> out[o] = in[2o] + ext, eval form throughout.
// cur: [count*2][2][n]; nxt: [count][2][n]; the RGSW of CMux o ([2L][2][n],
// eval) is picked by `ks`. The digits never leave registers. Every transform
// and RGSW product is exact integer arithmetic on doubles (ntt_fp.cuh: FMA
// two-products and a floating-point quotient estimate). For single primes
// q < 2^35 and small gadgets: differences of canonical residues are
// below q; the inverse leaves coefficients within 0.5625 q, made canonical for
// the digit split; digits below B/2 transform to values below 7 q; each product
// with an RGSW sample (below q) is reduced to within 0.5625 q, so the 2L
// products and the input residue sum to less than (1 + 1.125 L) q before the
// final reduction.
template <int LOGN>
__global__ void __launch_bounds__((1 << LOGN) / 8, LOGN >= 12 ? 1 : 2) k_cmux_fp(const u64* __restrict__ cur,
                                                                                u64* __restrict__ nxt, KeySel ks,
                                                                                DevRing R, Gadget g) {
  constexpr int n = 1 << LOGN;
  using In0 = NttPhase<LOGN, true, 0>;
  using InL = NttPhase<LOGN, true, (LOGN + 2) / 3 - 1>;
  using Fw0 = NttPhase<LOGN, false, 0>;
  using FwL = NttPhase<LOGN, false, (LOGN + 2) / 3 - 1>;
  static_assert(In0::STRIDE == 1 && In0::R == 3 && FwL::STRIDE == 1, "contiguous end layouts");
  __shared__ double ssm[n];
  const int tid = threadIdx.x;
  const long o = blockIdx.x;
  const NttTable& T = R.t[0];
  const double q = T.qd, qinv = T.qinv;
  const u64* a = cur + (2 * o) * 2 * n;
  const u64* b = a + 2 * n;
  const u64* K = ks.base + ((o / ks.div) % ks.mod) * ks.stride;
  const int L = g.L;
  double am[8], ab[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) am[v] = ab[v] = 0.0;
  for (int p = 0; p < 2; ++p) {  // 0: mask digits (neg_s_m rows), 1: body digits (m rows)
    double e[8];
    {
      const ulonglong2* bv = reinterpret_cast<const ulonglong2*>(b + p * n + 8 * tid);
      const ulonglong2* av = reinterpret_cast<const ulonglong2*>(a + p * n + 8 * tid);
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const ulonglong2 x = bv[h], y = av[h];
        e[2 * h] = __dadd_rn(__ull2double_rn(x.x), -__ull2double_rn(y.x));
        e[2 * h + 1] = __dadd_rn(__ull2double_rn(x.y), -__ull2double_rn(y.y));
      }
    }
    ntt_inverse_fp<LOGN>(e, tid, T, ssm);
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 8; ++v) ssm[swz(InL::index(v, tid))] = e[v];
    __syncthreads();
    u32 dcur[8];  // scaled coefficients, below B^L < 2^32
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      double c = ssm[swz(Fw0::index(v, tid))];
      if (c < 0.0) c = __dadd_rn(c, q);
      dcur[v] = (u32)gadget_scaled_small((u64)__double2ull_rn(c), g);
    }
    for (int k = 0; k < L; ++k) {
#pragma unroll
      for (int v = 0; v < 8; ++v) e[v] = __ll2double_rn(gadget_next_digit32(dcur[v], g));
      ntt_forward_fp<LOGN>(e, tid, T, ssm);
      const ulonglong2* Km = reinterpret_cast<const ulonglong2*>(K + (long)(2 * (p * L + L - 1 - k)) * n + 8 * tid);
      const ulonglong2* Kb = Km + n / 2;
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const ulonglong2 km = __ldg(Km + h), kb = __ldg(Kb + h);
        am[2 * h] = __dadd_rn(am[2 * h], fp_mulmod(e[2 * h], __ull2double_rn(km.x), q, qinv));
        am[2 * h + 1] = __dadd_rn(am[2 * h + 1], fp_mulmod(e[2 * h + 1], __ull2double_rn(km.y), q, qinv));
        ab[2 * h] = __dadd_rn(ab[2 * h], fp_mulmod(e[2 * h], __ull2double_rn(kb.x), q, qinv));
        ab[2 * h + 1] = __dadd_rn(ab[2 * h + 1], fp_mulmod(e[2 * h + 1], __ull2double_rn(kb.y), q, qinv));
      }
    }
  }
  ulonglong2* outm = reinterpret_cast<ulonglong2*>(nxt + o * 2 * n + 8 * tid);
  ulonglong2* outb = outm + n / 2;
  const ulonglong2* am_in = reinterpret_cast<const ulonglong2*>(a + 8 * tid);
  const ulonglong2* ab_in = am_in + n / 2;
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const ulonglong2 xm = am_in[h], xb = ab_in[h];
    ulonglong2 ym, yb;
    ym.x = __double2ull_rn(fp_canonical(__dadd_rn(__ull2double_rn(xm.x), am[2 * h]), q, qinv));
    ym.y = __double2ull_rn(fp_canonical(__dadd_rn(__ull2double_rn(xm.y), am[2 * h + 1]), q, qinv));
    yb.x = __double2ull_rn(fp_canonical(__dadd_rn(__ull2double_rn(xb.x), ab[2 * h]), q, qinv));
    yb.y = __double2ull_rn(fp_canonical(__dadd_rn(__ull2double_rn(xb.y), ab[2 * h + 1]), q, qinv));
    outm[h] = ym;
    outb[h] = yb;
  }
}

// The CMux of k_cmux_fp split over a cluster of four CTAs, for tree levels
// with too few CMuxes to fill the GPU, where one CMux's latency sets the level's
// time. CTA r of the cluster takes input half p = r & 1 (mask or body),
// inverse-transforms its difference, and forward-transforms its digit k = r >> 1;
// its products with the sample's mask and body (sample p L + L - 1 - k) are
// reduced mod q into its shared memory. After a cluster barrier, ranks 0 and 1
// add in[2o] and the four partial masks / bodies, read over distributed shared
// memory; a second barrier keeps every CTA's shared memory alive until those
// reads are done. Two transforms per CTA instead of six for one CTA. L = 2 and
// n <= 2048 (48 KB of static shared memory).
// In double precision with the bounds of k_cmux_fp: each CTA's products are
// signed residues within 0.5625 q, kept as doubles in shared memory; ranks 0
// and 1 add the four partials to in[2o] and reduce once.
template <int LOGN>
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__((1 << LOGN) / 8, 2)
    k_cmux_cluster_fp(const u64* __restrict__ cur, u64* __restrict__ nxt, KeySel ks, DevRing R, Gadget g) {
  namespace cg = cooperative_groups;
  constexpr int n = 1 << LOGN;
  using InL = NttPhase<LOGN, true, (LOGN + 2) / 3 - 1>;
  using Fw0 = NttPhase<LOGN, false, 0>;
  __shared__ double ssm[n];    // transform exchanges, then the mask partial
  __shared__ double pbody[n];  // the body partial
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  const int p = r & 1, k = r >> 1;
  const int tid = threadIdx.x;
  const long o = blockIdx.x / 4;
  const NttTable& T = R.t[0];
  const double q = T.qd, qinv = T.qinv;
  const u64* a = cur + (2 * o) * 2 * n;
  const u64* b = a + 2 * n;
  const u64* K = ks.base + ((o / ks.div) % ks.mod) * ks.stride;
  double e[8];
  {
    const ulonglong2* bv = reinterpret_cast<const ulonglong2*>(b + p * n + 8 * tid);
    const ulonglong2* av = reinterpret_cast<const ulonglong2*>(a + p * n + 8 * tid);
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const ulonglong2 x = bv[h], y = av[h];
      e[2 * h] = __dadd_rn(__ull2double_rn(x.x), -__ull2double_rn(y.x));
      e[2 * h + 1] = __dadd_rn(__ull2double_rn(x.y), -__ull2double_rn(y.y));
    }
  }
  ntt_inverse_fp<LOGN>(e, tid, T, ssm);
  __syncthreads();
#pragma unroll
  for (int v = 0; v < 8; ++v) ssm[swz(InL::index(v, tid))] = e[v];
  __syncthreads();
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    double c = ssm[swz(Fw0::index(v, tid))];
    if (c < 0.0) c = __dadd_rn(c, q);
    u32 sc = (u32)gadget_scaled_small((u64)__double2ull_rn(c), g);
    i64 d = gadget_next_digit32(sc, g);
    if (k) d = gadget_next_digit32(sc, g);
    e[v] = __ll2double_rn(d);
  }
  ntt_forward_fp<LOGN>(e, tid, T, ssm);
  const int smp = p * 2 + 1 - k;  // sample L - 1 - k of half p (L = 2)
  const ulonglong2* Km = reinterpret_cast<const ulonglong2*>(K + (long)(2 * smp) * n + 8 * tid);
  const ulonglong2* Kb = Km + n / 2;
  __syncthreads();  // every thread is done with the transform's exchanges in ssm
#pragma unroll
  for (int h = 0; h < 4; ++h) {
    const ulonglong2 km = __ldg(Km + h), kb = __ldg(Kb + h);
    const int s0 = 8 * tid + 2 * h;
    ssm[s0] = fp_mulmod(e[2 * h], __ull2double_rn(km.x), q, qinv);
    ssm[s0 + 1] = fp_mulmod(e[2 * h + 1], __ull2double_rn(km.y), q, qinv);
    pbody[s0] = fp_mulmod(e[2 * h], __ull2double_rn(kb.x), q, qinv);
    pbody[s0 + 1] = fp_mulmod(e[2 * h + 1], __ull2double_rn(kb.y), q, qinv);
  }
  cluster.sync();
  if (r < 2) {  // rank 0: the output mask, rank 1: the output body
    double* parts[4];
#pragma unroll
    for (int rr = 0; rr < 4; ++rr) parts[rr] = cluster.map_shared_rank(r == 0 ? ssm : pbody, rr);
    u64* out = nxt + o * 2 * n + (long)r * n;
    for (int x = tid; x < n; x += blockDim.x) {
      double acc = __ull2double_rn(a[(long)r * n + x]);
#pragma unroll
      for (int rr = 0; rr < 4; ++rr) acc = __dadd_rn(acc, parts[rr][x]);
      out[x] = __double2ull_rn(fp_canonical(acc, q, qinv));
    }
  }
  cluster.sync();
}

// CMux level o < count: fused kernel when the ring has one NTT limb of a
// supported degree and a small gadget, else diff -> external product -> add.
static bool cmux_fused_ok(const DevRing& R, const Gadget& g) {
  return R.ntt && R.nl == 1 && g.small && g.S < ((u128)1 << 32) && R.m[0].q < (1ull << 35) &&
         (R.n == 4096 || R.n == 2048 || R.n == 1024 || R.n == 512);
}

static void cmux_fused(const DevRing& R, const Gadget& g, const u64* cur, u64* nxt, KeySel ks, long count,
                       cudaStream_t st) {
  // Levels of at most 64 CMuxes leave most SMs idle: split each CMux over a
  // four-CTA cluster to cut its latency.
  if (count <= 64 && g.L == 2 && R.n <= 2048) {
    switch (R.n) {
      case 2048: k_cmux_cluster_fp<11><<<(unsigned)(4 * count), 256, 0, st>>>(cur, nxt, ks, R, g); break;
      case 1024: k_cmux_cluster_fp<10><<<(unsigned)(4 * count), 128, 0, st>>>(cur, nxt, ks, R, g); break;
      default: k_cmux_cluster_fp<9><<<(unsigned)(4 * count), 64, 0, st>>>(cur, nxt, ks, R, g); break;
    }
    VIA_LAUNCHED();
    return;
  }
  switch (R.n) {
    case 4096: k_cmux_fp<12><<<(unsigned)count, 512, 0, st>>>(cur, nxt, ks, R, g); break;
    case 2048: k_cmux_fp<11><<<(unsigned)count, 256, 0, st>>>(cur, nxt, ks, R, g); break;
    case 1024: k_cmux_fp<10><<<(unsigned)count, 128, 0, st>>>(cur, nxt, ks, R, g); break;
    default: k_cmux_fp<9><<<(unsigned)count, 64, 0, st>>>(cur, nxt, ks, R, g); break;
  }
  VIA_LAUNCHED();
}

// CRot diff for nq RLWEs: rot = -(X^k * ct), diff = rot - ct.
__global__ void k_crot_diff_batch(const u64* ct, int n, int k, long nq, DevMod m, u64* diff) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nq * 2 * n) return;
  long p = gid / n;
  int i = (int)(gid % n);
  int src = i - k;
  bool wrap = src < 0;
  if (wrap) src += n;
  u64 v = ct[p * n + src];
  u64 xk = wrap ? negmod(v, m.q) : v;
  diff[p * n + i] = submod(negmod(xk, m.q), ct[p * n + i], m.q);
}

__global__ void k_ring_switch_proj_batch(const u64* ct, int n1, int n2, long nq, DevMod m, u64* mask_proj,
                                         u64* body_proj) {
  const int d = n1 / n2;
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nq * (d + 1) * n2) return;
  long q = gid / ((d + 1) * n2);
  int r = (int)(gid % ((d + 1) * n2));
  int j = r / n2, t = r % n2;
  const u64* c = ct + q * 2 * n1;
  if (j == d) {
    body_proj[q * n2 + t] = c[n1 + d * t];
    return;
  }
  int src = d * t - j;
  bool wrap = src < 0;
  if (wrap) src += n1;
  u64 v = c[src];
  mask_proj[(q * d + j) * n2 + t] = wrap ? negmod(v, m.q) : v;
}

__global__ void k_ring_switch_sum_batch(const u64* gp, int d, int n2, long nq, DevMod m, u64* acc) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nq * 2 * n2) return;
  long q = gid / (2 * n2);
  int r = (int)(gid % (2 * n2));
  int mb = r / n2, t = r % n2;
  u64 sacc = 0;
  for (int j = 0; j < d; ++j) sacc = addmod(sacc, gp[((q * d + j) * 2 + mb) * n2 + t], m.q);
  acc[q * 2 * n2 + mb * n2 + t] = sacc;
}

__global__ void k_ring_switch_finish_batch(const u64* acc, const u64* body_proj, int n2, long nq, DevMod m3, DevMod m4,
                                           double dq3, u64* out_mask, u64* out_body) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nq * n2) return;
  long q = gid / n2;
  int t = (int)(gid % n2);
  const u64 q3 = m3.q;
  const u64* a = acc + q * 2 * n2;
  out_mask[q * n2 + t] = negmod(a[t], q3);  // mask: q3 -> q3 is the identity rescale
  u64 body = submod(body_proj[q * n2 + t], a[n2 + t], q3);
  // body: q3 -> q4 (mod_switch_asym, prim/switching/mod_switch.rs:124-154).
  u128 num = (u128)body * m4.q + q3 / 2;
  u64 r = (u64)div_exact(num, (u128)q3, dq3);
  out_body[q * n2 + t] = r >= m4.q ? r - m4.q : r;
}

// Step 7, RespComp (resp_comp.rs:46-76), of B RLWEs at (q2, n1) in coefficient
// form: q2 -> q3, ring switch n1 -> n2 with the RSK, body q3 -> q4.
static void resp_comp(Server& s, Workspace& w, const u64* ct_q2, long B, u64* d_mask, u64* d_body,
                      cudaStream_t st) {
  const via_params& p = s.prm;
  const int n1 = p.n1, n2 = p.n2;
  mod_switch(s.r2, ct_q2, s.r3n1, w.rs_ct3.p, B * 2, n1, st);
  const int d = n1 / n2;
  k_ring_switch_proj_batch<<<blocks(B * (d + 1) * n2), 256, 0, st>>>(w.rs_ct3.p, n1, n2, B, s.r3.m[0], w.rs_mproj.p,
                                                                      w.rs_bproj.p);
  VIA_LAUNCHED();
  gadget_product(s.r3, w.g_rsk, w.rs_mproj.p, n2, 1, 1, B * d, keys_cyclic(s.rsk_eval.p, d), w.rs_gp.p,
                 w.rs_digits.p, st);
  k_ring_switch_sum_batch<<<blocks(B * 2 * n2), 256, 0, st>>>(w.rs_gp.p, d, n2, B, s.r3.m[0], w.rs_acc.p);
  VIA_LAUNCHED();
  from_eval(s.r3, w.rs_acc.p, n2, B * 2, st);
  k_ring_switch_finish_batch<<<blocks(B * n2), 256, 0, st>>>(w.rs_acc.p, w.rs_bproj.p, n2, B, s.r3.m[0], s.r4.m[0],
                                                             (double)p.q3, d_mask, d_body);
  VIA_LAUNCHED();
}

// Runs the pipeline for nq queries (d_query: nq queries back to back; d_mask,
// d_body: [nq][n2]). When stop_stage > 0 (nq == 1 only), copies that stage's
// output in coefficient form to `dump` and returns early. Stages: 1 cascade
// RLWEs, 2 query RGSWs at q1, 3 DMux outputs, 4 mod-switched rows at q2,
// 5 FirstDim columns, 6 CMux output, 7 CRot output.
void answer_device_stages(Server& s, Workspace& w, const u64* d_query, int nq, u64* d_mask, u64* d_body,
                          cudaStream_t st, int stop_stage, u64* dump) {
  const via_params& p = s.prm;
  const int n1 = p.n1, L = p.l_query, nl = s.r1.nl;
  const long I = p.num_rows, J = p.num_cols, B = nq;
  const int nd = ilog2(I), nc = ilog2(J);
  const int nr = (int)(w.nbits - nd - nc);
  const long rgsw1 = 2L * L * 2 * nl * n1, rgsw2 = 2L * L * 2 * n1;
  if (nq < 1 || nq > w.bmax) throw CudaError(100, "batch larger than the workspace");
  auto copy_out = [&](const u64* src, size_t count) {
    VIA_CUDA(cudaMemcpyAsync(dump, src, count * 8, cudaMemcpyDeviceToDevice, st));
  };
  // ---- Step 1: QueryDecomp. The LWEs are taken grouped by use (every query's
  // DMux bits, then every query's CMux and CRot bits), so the RGSWs come out in
  // the grouped layout of rgsw_q1 and each group is one contiguous range.
  const long nb = w.nbits - nd;                 // CMux + CRot bits per query
  const long lwe_a = (long)nd * L, nlwe_all = w.nlwe * B;
  const u64* qsrc = d_query;
  if (B > 1) {
    const long ll = (long)lwe_len(p);
    k_permute_lwes<<<blocks(nlwe_all * ll), 256, 0, st>>>(d_query, B, w.nlwe, lwe_a, ll, w.q_perm.p);
    VIA_LAUNCHED();
    qsrc = w.q_perm.p;
  }
  u64* const rgsw_b1 = w.rgsw_q1.p + B * nd * rgsw1;  // the CMux / CRot bits' group
  u64* const rgsw_b2 = w.rgsw_q2.p + B * nd * rgsw2;
  // Answers that run to the end expand the CMux / CRot bits (their cascades,
  // RGSWs and q1 -> q2 switch) on the side stream while the DMux tree and the
  // database scan run on `st`; `st` waits for them before the CMux tree. The
  // two groups' LWEs, buffer regions and scratch are disjoint.
  const bool split = (stop_stage == 0 || stop_stage == STOP_AFTER_CROT) && nd > 0 && nb > 0 && s.r1.ntt;
  if (split) {
    VIA_CUDA(cudaEventRecord(w.ev_fork, st));
    VIA_CUDA(cudaStreamWaitEvent(w.side, w.ev_fork, 0));
    query_decomp_range(s, w, qsrc, B * lwe_a, nlwe_all - B * lwe_a, B * nd, B * nb, w.side);
    mod_switch(s.r1, rgsw_b1, s.r2, rgsw_b2, B * nb * 2 * L * 2, n1, w.side);
    to_eval(s.r2, rgsw_b2, n1, B * nb * 2 * L * 2, w.side);
    VIA_CUDA(cudaEventRecord(w.ev_join, w.side));
    query_decomp_range(s, w, qsrc, 0, B * lwe_a, 0, B * nd, st);
    to_eval(s.r1, w.rgsw_q1.p, n1, B * nd * 2 * L * 2 * nl, st);
  } else {
    query_decomp_range(s, w, qsrc, 0, nlwe_all, 0, B * w.nbits, st);
    if (stop_stage == 1) return copy_out(w.c_rlwe.p, (size_t)w.nlwe * 2 * nl * n1);
    if (stop_stage == 2) return copy_out(w.rgsw_q1.p, (size_t)w.nbits * rgsw1);  // one query: bit order

    // ---- mod_switch_rgsw q1 -> q2 of every bit (convert.rs:223-240; only the
    // CMux / CRot bits are used at q2), then eval form for both moduli.
    mod_switch(s.r1, w.rgsw_q1.p, s.r2, w.rgsw_q2.p, B * w.nbits * 2 * L * 2, n1, st);
    to_eval(s.r2, w.rgsw_q2.p, n1, B * w.nbits * 2 * L * 2, st);
    to_eval(s.r1, w.rgsw_q1.p, n1, B * w.nbits * 2 * L * 2 * nl, st);
  }

  // ---- Step 2: DMux tree at q1 from the trivial RLWE(0, delta) (answer.rs:181-191).
  {
    u128 Q1 = s.r1.Q();
    u128 delta = (Q1 + p.p - 1) / p.p;
    k_set_trivial<<<blocks(B * 2 * nl * n1), 256, 0, st>>>(w.dm_a.p, B, n1, nl, (u64)(delta % s.r1.m[0].q),
                                                           (u64)(delta % s.r1.m[1].q));
    VIA_LAUNCHED();
    u64 *in = w.dm_a.p, *out = w.dm_b.p;
    for (int i = 0; i < nd; ++i) {
      const long active = 1L << i;  // per query
      KeySel bit{w.rgsw_q1.p + i * rgsw1, active, B, nd * rgsw1};
      // The fused level kernel is latency-bound at about 70 us for up to a wave of
      // products (148 SMs x 2 CTAs, two per product); smaller levels keep the
      // separate, wider kernels (about 40 us a level).
      if (dmux_fp_ok(s.r1, w.g_dmux) && B * active >= 256) {
        k_dmux_fp<11><<<dim3((unsigned)(B * active), 2), 256, 0, st>>>(out, in, bit, s.r1, w.g_dmux);
        VIA_LAUNCHED();
        std::swap(in, out);
        continue;
      }
      if (R_fp_small(s.r1)) {
        external_products(s.r1, w.g_dmux, bit, in, B * active, w.dm_digits.p, w.dm_ext.p, false, st);
        intt_epi<INTT_DMUX>(s.r1, w.dm_ext.p, in, out, B * active, st);
        std::swap(in, out);
        continue;
      }
      external_products(s.r1, w.g_dmux, bit, in, B * active, w.dm_digits.p, w.dm_ext.p, true, st);
      k_dmux_combine<<<blocks(B * active * 2 * nl * n1), 256, 0, st>>>(out, in, w.dm_ext.p, B * active, n1, nl, s.r1);
      VIA_LAUNCHED();
      std::swap(in, out);
    }
    if (stop_stage == 3) return copy_out(in, (size_t)I * 2 * nl * n1);
    // ---- Step 3: ModSwitch q1 -> q2 (answer.rs:194-199) into the selection rows.
    mod_switch(s.r1, in, s.r2, w.sel.p, B * 2 * I, n1, st);
  }
  if (stop_stage == 4) return copy_out(w.sel.p, (size_t)I * 2 * n1);

  // ---- Step 4: FirstDim (answer.rs:204-205), one pass over the database for
  // the whole batch; the columns stay in the eval domain.
  to_eval(s.r2, w.sel.p, n1, B * 2 * I, st);
  first_dim_queries(s, w.sel.p, w.fd_out.p, nq, reinterpret_cast<uint8_t*>(w.sel_bytes.p), st);
  if (stop_stage == 5) {
    copy_out(w.fd_out.p, (size_t)J * 2 * n1);
    from_eval(s.r2, dump, n1, 2 * J, st);
    return;
  }

  if (split) VIA_CUDA(cudaStreamWaitEvent(st, w.ev_join, 0));  // the CMux / CRot RGSWs are ready

  // ---- Step 5: CMux tree (mux.rs:167-198), level by level in the eval domain:
  // diff = in[2j+1] - in[2j] (eval) -> coeff -> gadget product -> out[j] = in[2j] + ext.
  u64* cur = w.fd_out.p;
  for (int i = 0; i < nc; ++i) {
    const long half = (J >> i) / 2;  // CMuxes per query at this level
    KeySel bit{rgsw_b2 + i * rgsw2, half, B, nb * rgsw2};
    u64* nxt = cur == w.fd_out.p ? w.cm_b.p : w.fd_out.p;  // ping-pong between fd_out and cm_b
    if (cmux_fused_ok(s.r2, w.g_cmux)) {
      cmux_fused(s.r2, w.g_cmux, cur, nxt, bit, B * half, st);
      cur = nxt;
      continue;
    }
    k_rlwe_addsub<<<blocks(B * half * 2 * n1), 256, 0, st>>>(w.cm_diff.p, cur + 2 * n1, 2, cur, 2, -1, B * half, n1, 1,
                                                             s.r2);
    VIA_LAUNCHED();
    from_eval(s.r2, w.cm_diff.p, n1, B * 2 * half, st);
    external_products(s.r2, w.g_cmux, bit, w.cm_diff.p, B * half, w.cm_digits.p, w.cm_ext.p, false, st);
    k_rlwe_addsub<<<blocks(B * half * 2 * n1), 256, 0, st>>>(nxt, cur, 2, w.cm_ext.p, 1, +1, B * half, n1, 1, s.r2);
    VIA_LAUNCHED();
    cur = nxt;
  }
  // Selected columns back to coefficient form.
  if (!intt_epi<INTT_STORE>(s.r2, cur, nullptr, w.cr_ct.p, B, st)) {
    VIA_CUDA(cudaMemcpyAsync(w.cr_ct.p, cur, (size_t)B * 2 * n1 * 8, cudaMemcpyDeviceToDevice, st));
    from_eval(s.r2, w.cr_ct.p, n1, B * 2, st);
  }
  if (stop_stage == 6) return copy_out(w.cr_ct.p, 2 * (size_t)n1);

  // ---- Step 6: CRot, SlotExtract (rotate.rs:128-150).
  for (int i = 0; i < nr; ++i) {
    k_crot_diff_batch<<<blocks(B * 2 * n1), 256, 0, st>>>(w.cr_ct.p, n1, n1 - (1 << i), B, s.r2.m[0], w.cr_diff.p);
    VIA_LAUNCHED();
    KeySel bit{rgsw_b2 + (nc + i) * rgsw2, 1, B, nb * rgsw2};
    if (R_fp_small(s.r2)) {
      external_products(s.r2, w.g_cmux, bit, w.cr_diff.p, B, w.cr_digits.p, w.cr_ext.p, false, st);
      intt_epi<INTT_ADD>(s.r2, w.cr_ext.p, w.cr_ct.p, w.cr_ct.p, B, st);
      continue;
    }
    external_products(s.r2, w.g_cmux, bit, w.cr_diff.p, B, w.cr_digits.p, w.cr_ext.p, true, st);
    k_rlwe_addsub<<<blocks(B * 2 * n1), 256, 0, st>>>(w.cr_ct.p, w.cr_ct.p, 1, w.cr_ext.p, 1, +1, B, n1, 1, s.r2);
    VIA_LAUNCHED();
  }
  if (stop_stage == 7) return copy_out(w.cr_ct.p, 2 * (size_t)n1);
  if (stop_stage == STOP_AFTER_CROT) return;
  resp_comp(s, w, w.cr_ct.p, B, d_mask, d_body, st);
}

void answer_device_stages(Server& s, const u64* d_query, int nq, u64* d_mask, u64* d_body, cudaStream_t st,
                          int stop_stage, u64* dump) {
  answer_device_stages(s, *s.ws, d_query, nq, d_mask, d_body, st, stop_stage, dump);
}

void answer_device(Server& s, const u64* d_query, u64* d_mask, u64* d_body, cudaStream_t st) {
  answer_device_stages(s, d_query, 1, d_mask, d_body, st, 0, nullptr);
}

u64* ws_query(Workspace& w) { return w.q_in.p; }
u64* ws_answer_mask(Workspace& w) { return w.a_mask.p; }
u64* ws_answer_body(Workspace& w) { return w.a_body.p; }
u64* workspace_query(Server& s) { return s.ws->q_in.p; }
u64* workspace_answer_mask(Server& s) { return s.ws->a_mask.p; }
u64* workspace_answer_body(Server& s) { return s.ws->a_body.p; }

// The whole answer for nq queries (~220 kernels) on the workspace buffers,
// captured once per batch size into a CUDA graph and replayed.
// st == nullptr captures (if needed) without launching.
void answer_graph(Server& s, Workspace& w, int nq, cudaStream_t st) {
  cudaGraphExec_t exec = nullptr;
  unsigned long long kernels = 0;
  if (w.graphs_gen != s.plan_gen) {  // the scan tiles changed since these were captured
    for (auto& g : w.graphs) cudaGraphExecDestroy(g.second);
    w.graphs.clear();
    w.graph_kernels.clear();
    w.graphs_gen = s.plan_gen;
  }
  for (size_t i = 0; i < w.graphs.size(); ++i)
    if (w.graphs[i].first == nq) {
      exec = w.graphs[i].second;
      kernels = w.graph_kernels[i].second;
    }
  if (!exec) {
    cudaGraph_t g;
    unsigned long long before = __atomic_load_n(&g_kernel_launches, __ATOMIC_RELAXED);
    VIA_CUDA(cudaStreamBeginCapture(w.capture, cudaStreamCaptureModeThreadLocal));
    try {
      answer_device_stages(s, w, w.q_in.p, nq, w.a_mask.p, w.a_body.p, w.capture, 0, nullptr);
    } catch (...) {
      cudaStreamEndCapture(w.capture, &g);
      throw;
    }
    VIA_CUDA(cudaStreamEndCapture(w.capture, &g));
    kernels = __atomic_load_n(&g_kernel_launches, __ATOMIC_RELAXED) - before;
    __atomic_sub_fetch(&g_kernel_launches, kernels, __ATOMIC_RELAXED);  // captured, not run
    cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    VIA_CUDA(e);
    w.graphs.push_back({nq, exec});
    w.graph_kernels.push_back({nq, kernels});
  }
  if (!st) return;
  VIA_CUDA(cudaGraphLaunch(exec, st));
  __atomic_add_fetch(&g_kernel_launches, kernels, __ATOMIC_RELAXED);
}

void answer_graph(Server& s, int nq, cudaStream_t st) { answer_graph(s, *s.ws, nq, st ? st : s.stream); }


// ===========================================================================
// VIA-B: repack of T CRot outputs into one RLWE (crates/via-primitives/src/
// conversion/repack.rs, crates/via-server/src/batch.rs:72-163).
//
// A level's list of MLWEs is stored as masks [count][rank][deg] and bodies
// [count][deg] at q2, coefficient form. Extr_{n_rec} turns each CRot output into
// an (n1/n_rec, n_rec)-MLWE; input t goes to position bitrev(t) (the reference
// swaps the T inputs into bit-reversed order) and positions >= T are zero
// MLWEs. Each level pairs entries (2p, 2p+1): embed_d interleaves the pair
// (slots 0 and 1), every embedded mask is key-switched with the level's
// q2-switched cascade keys, and conv_step's slot reduction gives
// masks_out[j] = -(P[j].mask + P[j+R/2].mask), body = embed_d(bodies) - sum P.body.
// Pairs of two zero MLWEs give zero MLWEs (zero digits), so only the leading
// nonzero entries are processed.
// ===========================================================================

// masks/bodies of the level-0 list from the CRot outputs ct [T][2][n1].
__global__ void k_repack_extr(const u64* __restrict__ ct, int T, int lt, int n1, int g, DevMod m, u64* __restrict__ masks,
                              u64* __restrict__ bodies) {
  const int D = n1 / g;
  const long total = (long)T * (D + 1) * g;
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= total) return;
  const int i = (int)(gid % g);
  const int k = (int)((gid / g) % (D + 1));
  const int t = (int)(gid / ((long)g * (D + 1)));
  int pos = 0;
  for (int b = 0; b < lt; ++b) pos |= ((t >> b) & 1) << (lt - 1 - b);
  const u64* mask = ct + (long)t * 2 * n1;
  const u64* body = mask + n1;
  if (k == D) {
    bodies[(long)pos * g + i] = body[(long)D * i];
    return;
  }
  u64 v;
  if (k == 0) {
    v = mask[(long)D * i];
  } else {
    // (X * pi_{D-k}(A))[i]: pi[i-1], and -pi[g-1] at i = 0.
    const int slot = D - k;
    v = i == 0 ? negmod(mask[(long)D * (g - 1) + slot], m.q) : mask[(long)D * (i - 1) + slot];
  }
  masks[((long)pos * D + k) * g + i] = v;
}

// embed_d (d = 2) of `pairs` pairs: emb_masks [pair][rank][2 n_in], emb_body [pair][2 n_in].
__global__ void k_repack_embed(const u64* __restrict__ masks, const u64* __restrict__ bodies, long pairs, int rank,
                               int n_in, u64* __restrict__ emb_masks, u64* __restrict__ emb_body) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= pairs * (rank + 1) * n_in) return;
  const int i = (int)(gid % n_in);
  const int k = (int)((gid / n_in) % (rank + 1));
  const long pr = gid / ((long)n_in * (rank + 1));
  const int n_out = 2 * n_in;
  if (k == rank) {
    emb_body[pr * n_out + 2 * i] = bodies[(2 * pr) * n_in + i];
    emb_body[pr * n_out + 2 * i + 1] = bodies[(2 * pr + 1) * n_in + i];
    return;
  }
  u64* o = emb_masks + (pr * rank + k) * n_out;
  o[2 * i] = masks[((2 * pr) * rank + k) * n_in + i];
  o[2 * i + 1] = masks[((2 * pr + 1) * rank + k) * n_in + i];
}

__global__ void k_sub_polys(const u64* __restrict__ a, const u64* __restrict__ b, long count, DevMod m,
                            u64* __restrict__ out) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= count) return;
  out[gid] = submod(a[gid], b[gid], m.q);
}

// The repack keys: for every output degree nout = 2 n_rec .. n1 the cascade step
// of that degree (rank_in = 2 n1 / nout RLevs of L_CK samples), switched from q1
// to q2 sample by sample (mod_switch_rlev, repack.rs:684-739) and transformed at
// q2. Must run before the cascade key itself is transformed.
void derive_repack_keys(Server& s) {
  const via_params& p = s.prm;
  if (via_b_batch(p) < 2 || !s.cascade_eval.p) return;
  const int n1 = p.n1, L = p.l_ck, nl = s.r1.nl;
  const u64 step_len = (u64)2 * n1 * L * 2 * nl;
  size_t total = 0;
  s.repack_off.clear();
  for (int nout = 2 * (int)p.n_rec; nout <= n1; nout <<= 1) {
    s.repack_off.push_back(total);
    total += (size_t)(2 * n1 / nout) * L * 2 * nout;
  }
  s.repack_eval.alloc(total);
  int level = 0;
  for (int nout = 2 * (int)p.n_rec; nout <= n1; nout <<= 1, ++level) {
    const int k = ilog2(nout);  // cascade step k has output degree 2^k
    const long polys = (long)(2 * n1 / nout) * L * 2;
    u64* dst = s.repack_eval.p + s.repack_off[level];
    mod_switch(s.r1, s.cascade_eval.p + (k - 1) * step_len, s.r2, dst, polys, nout, s.stream);
    to_eval(s.r2, dst, nout, polys, s.stream);
  }
}

struct RepackWs {
  int T = 0;
  DevBuf la_m, la_b, lb_m, lb_b, emb_m, emb_b, digits, P, bsum, packed;
  DevBuf crot_all;  // CRot outputs of a batch run in chunks [T * groups][2][n1]
  Gadget g;
};

// Called with the workspace owned by the caller.
static RepackWs& repack_ws(Server& s, Workspace& w) {
  if (!w.repack) {
    const via_params& p = s.prm;
    auto r = std::make_unique<RepackWs>();
    const long T = via_b_batch(p), n1 = p.n1, L = p.l_ck;
    const long pairs = std::max(1L, T / 2);
    r->T = (int)T;
    // Level lists hold at most T (+1 zero partner) entries of n1 + deg residues.
    r->la_m.alloc((T + 2) * n1);
    r->la_b.alloc((T + 2) * n1);
    r->lb_m.alloc((T + 2) * n1);
    r->lb_b.alloc((T + 2) * n1);
    r->emb_m.alloc(pairs * 2 * n1);
    r->emb_b.alloc(pairs * n1);
    r->digits.alloc(pairs * 2 * n1 * L);
    r->P.alloc(pairs * 4 * n1);
    r->bsum.alloc(pairs * n1);
    r->g = make_gadget(p.ck_base, (int)p.l_ck, s.r2);
    if (T > w.bmax) r->crot_all.alloc(T * 2 * n1);  // one batch runs in chunks of bmax queries
    w.repack = std::move(r);
  }
  return *w.repack;
}

static void repack(Server& s, Workspace& w, const u64* crot, u64* out_rlwe, cudaStream_t st) {
  const via_params& p = s.prm;
  RepackWs& r = repack_ws(s, w);
  const int n1 = p.n1, g = (int)p.n_rec, T = r.T, D = n1 / g;
  int lt = 0;
  while ((1 << lt) < T) ++lt;
  u64 *cm = r.la_m.p, *cb = r.la_b.p, *nm = r.lb_m.p, *nb = r.lb_b.p;
  {
    const long total = (long)T * (D + 1) * g;
    k_repack_extr<<<blocks(total), 256, 0, st>>>(crot, T, lt, n1, g, s.r2.m[0], cm, cb);
    VIA_LAUNCHED();
  }
  long active = T;  // leading nonzero entries of the current list
  int rank = D, level = 0;
  for (int n_in = g; n_in < n1; n_in <<= 1, rank >>= 1, ++level) {
    const int n_out = 2 * n_in;
    if (active & 1) {  // the last pair's partner is a zero MLWE
      VIA_CUDA(cudaMemsetAsync(cm + active * rank * n_in, 0, (size_t)rank * n_in * 8, st));
      VIA_CUDA(cudaMemsetAsync(cb + active * n_in, 0, (size_t)n_in * 8, st));
    }
    const long pairs = (active + 1) / 2;
    k_repack_embed<<<blocks(pairs * (rank + 1) * n_in), 256, 0, st>>>(cm, cb, pairs, rank, n_in, r.emb_m.p, r.emb_b.p);
    VIA_LAUNCHED();
    gadget_product(s.r2, r.g, r.emb_m.p, n_out, 1, 1, pairs * rank,
                   keys_cyclic(s.repack_eval.p + s.repack_off[level], rank), r.P.p, r.digits.p, st);
    const long items = pairs * (rank / 2 + 1) * n_out;
    k_cascade_reduce<<<blocks(items), 256, 0, st>>>(r.P.p, rank, n_out, 1, pairs, s.r2, nm, r.bsum.p);
    VIA_LAUNCHED();
    from_eval(s.r2, nm, n_out, pairs * (rank / 2), st);
    from_eval(s.r2, r.bsum.p, n_out, pairs, st);
    k_sub_polys<<<blocks(pairs * n_out), 256, 0, st>>>(r.emb_b.p, r.bsum.p, pairs * n_out, s.r2.m[0], nb);
    VIA_LAUNCHED();
    std::swap(cm, nm);
    std::swap(cb, nb);
    active = pairs;
  }
  // The rank-1 MLWE of degree n1 is the RLWE (mask, body).
  VIA_CUDA(cudaMemcpyAsync(out_rlwe, cm, (size_t)n1 * 8, cudaMemcpyDeviceToDevice, st));
  VIA_CUDA(cudaMemcpyAsync(out_rlwe + n1, cb, (size_t)n1 * 8, cudaMemcpyDeviceToDevice, st));
}

// answer_batch (srv/batch.rs:72-163): the prefix through CRot for the T queries
// (sharing one database scan), the repack, and RespComp once.
// `groups` VIA-B batches of T queries each (d_queries back to back); answer g
// goes to d_mask/d_body + g * n2.
void answer_batch_device(Server& s, Workspace& w, const u64* d_queries, int groups, u64* d_mask, u64* d_body,
                         cudaStream_t st) {
  const int T = via_b_batch(s.prm);
  const int n1 = s.prm.n1;
  if (T < 2) throw CudaError(100, "answer_batch: the server was set up for VIA-C (n_rec = n2)");
  if (!s.repack_eval.p) throw CudaError(100, "answer_batch: no repack keys");
  RepackWs& r = repack_ws(s, w);
  const int total = T * groups;
  const u64* crot = w.cr_ct.p;
  if (total <= w.bmax) {
    answer_device_stages(s, w, d_queries, total, nullptr, nullptr, st, STOP_AFTER_CROT, nullptr);
  } else {
    // More queries than the workspace holds: the prefix runs in chunks of bmax
    // queries (each chunk shares one database scan) and the CRot outputs are
    // gathered for the repack. Memory stays that of a bmax-query workspace.
    if (r.crot_all.n < (size_t)total * 2 * n1) {
      VIA_CUDA(cudaStreamSynchronize(st));
      r.crot_all.alloc((size_t)total * 2 * n1);
    }
    const size_t qlen = (size_t)query_lwes(s.prm) * lwe_len(s.prm);
    for (int q0 = 0; q0 < total; q0 += w.bmax) {
      const int nc = std::min(w.bmax, total - q0);
      answer_device_stages(s, w, d_queries + (size_t)q0 * qlen, nc, nullptr, nullptr, st, STOP_AFTER_CROT, nullptr);
      VIA_CUDA(cudaMemcpyAsync(r.crot_all.p + (size_t)q0 * 2 * n1, w.cr_ct.p, (size_t)nc * 2 * n1 * 8,
                               cudaMemcpyDeviceToDevice, st));
    }
    crot = r.crot_all.p;
  }
  if (!r.packed.p || r.packed.n < (size_t)groups * 2 * n1) r.packed.alloc((size_t)groups * 2 * n1);
  for (int g = 0; g < groups; ++g)
    repack(s, w, crot + (size_t)g * T * 2 * n1, r.packed.p + (size_t)g * 2 * n1, st);
  resp_comp(s, w, r.packed.p, groups, d_mask, d_body, st);
}

void answer_batch_device(Server& s, const u64* d_queries, u64* d_mask, u64* d_body, cudaStream_t st) {
  answer_batch_device(s, *s.ws, d_queries, 1, d_mask, d_body, st);
}


// ===========================================================================
// Standalone primitives (the reference's own kernel-level operations, on
// caller buffers; coefficient form in and out).
// ===========================================================================

// External products ext[c] = rgsw[c] (x) ct[c] (crates/via-primitives/src/
// encryption/rgsw.rs:108-121): every RGSW is transformed once per call (the
// reference re-transforms its samples per call too, rlev.rs:211-219), then the
// mask and body digits meet the neg_s_m and m samples.
//   rgsw [count][2L][2][nl][n], cts/out [count][2][nl][n].
// Scratch: rgsw_eval (count * 2L * 2 * nl * n), digits (count * 2L * nl * n).
void prim_external_products(const DevRing& R, const Gadget& g, const u64* rgsw, const u64* cts, long count, u64* out,
                            u64* rgsw_eval, u64* digits, cudaStream_t st) {
  const long per = (long)R.nl * R.n;
  VIA_CUDA(cudaMemcpyAsync(rgsw_eval, rgsw, (size_t)count * 2 * g.L * 2 * per * 8, cudaMemcpyDeviceToDevice, st));
  to_eval(R, rgsw_eval, R.n, count * 2 * g.L * 2 * R.nl, st);
  external_products(R, g, KeySel{rgsw_eval, 1, count, 0}, cts, count, digits, out, true, st);
}

// X^k a (negacyclic) of mask and body, split into masks [count][nl][n] and
// bodies [count][nl][n] (element.rs:328, ops.rs:147-180).
__global__ void k_rotate_split(const u64* __restrict__ cts, const u64* __restrict__ shifts, long count, int n, int nl,
                               DevRing R, u64* __restrict__ masks, u64* __restrict__ bodies) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long per = (long)nl * n;
  if (gid >= count * 2 * per) return;
  const long c = gid / (2 * per);
  const int part = (int)((gid / per) % 2);
  const int l = (int)((gid % per) / n), i = (int)(gid % n);
  const u64 k = shifts[c] % (u64)(2 * n);
  const u64 v = cts[gid];
  const u64 pos = (u64)i + k;  // < 3n
  const int dst = (int)(pos % (u64)n);
  const bool neg = ((pos / (u64)n) & 1) != 0;
  const u64 q = R.m[l].q;
  u64* o = (part == 0 ? masks : bodies) + c * per + (long)l * n;
  o[dst] = neg && v ? q - v : v;
}

// out = (-prod.mask, body - prod.body) (keyswitch.rs:99-102).
__global__ void k_key_switch_finish(const u64* __restrict__ prod, const u64* __restrict__ bodies, long count, int n,
                                    int nl, DevRing R, u64* __restrict__ out) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long per = (long)nl * n;
  if (gid >= count * per) return;
  const long c = gid / per;
  const long r = gid % per;
  const int l = (int)(r / n);
  const u64 q = R.m[l].q;
  const u64 pm = prod[(2 * c) * per + r], pb = prod[(2 * c + 1) * per + r];
  out[(2 * c) * per + r] = pm ? q - pm : 0;
  out[(2 * c + 1) * per + r] = submod(bodies[c * per + r], pb, q);
}

// Key switches of rotated ciphertexts: out[c] = key_switch(K, X^{shift[c]} ct[c]).
//   key: RLev of L samples [L][2][nl][n] (coefficient form), shared by all.
// Scratch: key_eval (L * 2 * nl * n), masks/bodies (count * nl * n each),
// digits (count * L * nl * n), prod (count * 2 * nl * n).
void prim_key_switches(const DevRing& R, const Gadget& g, const u64* key, const u64* cts, const u64* shifts, long count,
                       u64* out, u64* key_eval, u64* masks, u64* bodies, u64* digits, u64* prod, cudaStream_t st) {
  const int n = R.n;
  const long per = (long)R.nl * n;
  VIA_CUDA(cudaMemcpyAsync(key_eval, key, (size_t)g.L * 2 * per * 8, cudaMemcpyDeviceToDevice, st));
  to_eval(R, key_eval, n, (long)g.L * 2 * R.nl, st);
  k_rotate_split<<<blocks(count * 2 * per), 256, 0, st>>>(cts, shifts, count, n, R.nl, R, masks, bodies);
  VIA_LAUNCHED();
  gadget_product(R, g, masks, n, 1, 1, count, keys_shared(key_eval), prod, digits, st);
  from_eval(R, prod, n, count * 2 * R.nl, st);
  k_key_switch_finish<<<blocks(count * per), 256, 0, st>>>(prod, bodies, count, n, R.nl, R, out);
  VIA_LAUNCHED();
}

}  // namespace via
