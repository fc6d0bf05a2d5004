// FirstDim — the database scan (crates/via-server/src/first_dim.rs:94-184).
//
//   c_j = sum_i sel_i (.) db[i][j]   for every column j, mask and body,
//
// computed pointwise in the eval domain at q2. The database is HBM-resident in
// eval form, one u64 per residue, laid out [i][j][t] (t = eval slot): a warp
// reads 512 contiguous bytes per (i, j) and each thread streams its columns with
// 16-byte loads.
//
// Exact products without 128-bit arithmetic: every selection residue s < q2 <
// 2^34 is split once per query into s = s0 + 2^17 s1 (s0, s1 < 2^17). Then
//   sum_i d s = X0 + 2^17 X1,  X_k = sum_i d s_k < I 2^51,
// two u64 accumulators per output, exact for I <= 4096, reduced mod q2 once.
#include "first_dim.cuh"

namespace via {

constexpr int FD_TPT = 2;  // eval slots per thread (one 16-byte load per column)
constexpr int FD_THREADS = 128;

// sel (I RLWEs, [I][2][n] u64 < 2^34) -> split halves [I][2][n] as (s0, s1).
__global__ void k_split_sel(const u64* __restrict__ sel, uint2* __restrict__ out, long count) {
  long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= count) return;
  u64 s = sel[g];
  out[g] = make_uint2((u32)(s & 0x1FFFF), (u32)(s >> 17));
}

// Exact sums of d*s0 and d*s1 (d < 2^34, s0, s1 < 2^17): each product is below
// 2^51, so I <= 4096 of them fit a u64. The compiler emits IMAD.WIDE.U32 on the
// low word of d and IMAD on the high word.
struct SplitAcc {
  u64 x0, x1;
};

__device__ __forceinline__ void split_mac(SplitAcc& acc, u64 d, uint2 s) {
  acc.x0 += d * (u64)s.x;
  acc.x1 += d * (u64)s.y;
}

__device__ __forceinline__ u64 split_reduce(const SplitAcc& a, const DevMod& m) {
  // x0 + 2^17 x1 as 128 bits.
  u64 lo = a.x0 + (a.x1 << 17);
  u64 hi = (a.x1 >> 47) + (lo < a.x0 ? 1 : 0);
  return reduce128(hi, lo, m);
}

template <int JPT>
__global__ void __launch_bounds__(FD_THREADS) k_first_dim_ntt(const u64* __restrict__ db, const uint2* __restrict__ sel,
                                                              u64* __restrict__ out, int I, int J, int n, DevMod m) {
  const int t = (blockIdx.x * FD_THREADS + threadIdx.x) * FD_TPT;
  const int j0 = blockIdx.y * JPT;
  if (t >= n) return;
  SplitAcc am[JPT][FD_TPT], ab[JPT][FD_TPT];
#pragma unroll
  for (int jj = 0; jj < JPT; ++jj)
#pragma unroll
    for (int k = 0; k < FD_TPT; ++k) am[jj][k] = ab[jj][k] = SplitAcc{0, 0};
  const size_t row_stride = (size_t)J * n;
  const u64* dbp = db + (size_t)j0 * n + t;
  const uint4* selp = reinterpret_cast<const uint4*>(sel + t);
  const size_t sel_stride = (size_t)n / 2;  // uint4 per poly (2 slots per uint4)
#pragma unroll 2
  for (int i = 0; i < I; ++i) {
    const uint4 sm = __ldg(selp + (size_t)(2 * i) * sel_stride);
    const uint4 sb = __ldg(selp + (size_t)(2 * i + 1) * sel_stride);
    ulonglong2 d[JPT];
#pragma unroll
    for (int jj = 0; jj < JPT; ++jj) d[jj] = __ldcs(reinterpret_cast<const ulonglong2*>(dbp + (size_t)jj * n));
#pragma unroll
    for (int jj = 0; jj < JPT; ++jj) {
      split_mac(am[jj][0], d[jj].x, make_uint2(sm.x, sm.y));
      split_mac(am[jj][1], d[jj].y, make_uint2(sm.z, sm.w));
      split_mac(ab[jj][0], d[jj].x, make_uint2(sb.x, sb.y));
      split_mac(ab[jj][1], d[jj].y, make_uint2(sb.z, sb.w));
    }
    dbp += row_stride;
  }
#pragma unroll
  for (int jj = 0; jj < JPT; ++jj) {
    u64* o = out + (size_t)(2 * (j0 + jj)) * n + t;
    ulonglong2 rm, rb;
    rm.x = split_reduce(am[jj][0], m);
    rm.y = split_reduce(am[jj][1], m);
    rb.x = split_reduce(ab[jj][0], m);
    rb.y = split_reduce(ab[jj][1], m);
    *reinterpret_cast<ulonglong2*>(o) = rm;
    *reinterpret_cast<ulonglong2*>(o + n) = rb;
  }
}

// Shared scan for a batch of queries: each thread streams one column for a
// pair of slots and applies it to Q queries' selection vectors, so every 16-byte
// database load feeds 4Q products. sel: [nq][I][2][n] split halves; out:
// [nq][J][2][n]. Grid z enumerates groups of Q queries.
template <int Q>
__global__ void __launch_bounds__(FD_THREADS) k_first_dim_multi(const u64* __restrict__ db, const uint2* __restrict__ sel,
                                                                u64* __restrict__ out, int I, int J, int n, int q0,
                                                                DevMod m) {
  const int t = (blockIdx.x * FD_THREADS + threadIdx.x) * FD_TPT;
  const int j = blockIdx.y;
  const int qb = q0 + blockIdx.z * Q;
  if (t >= n) return;
  SplitAcc am[Q][FD_TPT], ab[Q][FD_TPT];
#pragma unroll
  for (int a = 0; a < Q; ++a)
#pragma unroll
    for (int k = 0; k < FD_TPT; ++k) am[a][k] = ab[a][k] = SplitAcc{0, 0};
  const size_t row_stride = (size_t)J * n;
  const u64* dbp = db + (size_t)j * n + t;
  const size_t qstride = (size_t)I * 2 * n / 2;  // uint4 per query
  const uint4* selp = reinterpret_cast<const uint4*>(sel + t) + (size_t)qb * qstride;
  const size_t pstride = (size_t)n / 2;
  for (int i = 0; i < I; ++i) {
    const ulonglong2 d = __ldcs(reinterpret_cast<const ulonglong2*>(dbp));
#pragma unroll
    for (int a = 0; a < Q; ++a) {
      const uint4 sm = __ldg(selp + a * qstride + (size_t)(2 * i) * pstride);
      const uint4 sb = __ldg(selp + a * qstride + (size_t)(2 * i + 1) * pstride);
      split_mac(am[a][0], d.x, make_uint2(sm.x, sm.y));
      split_mac(am[a][1], d.y, make_uint2(sm.z, sm.w));
      split_mac(ab[a][0], d.x, make_uint2(sb.x, sb.y));
      split_mac(ab[a][1], d.y, make_uint2(sb.z, sb.w));
    }
    dbp += row_stride;
  }
#pragma unroll
  for (int a = 0; a < Q; ++a) {
    u64* o = out + ((size_t)(qb + a) * J * 2 + 2 * (size_t)j) * n + t;
    ulonglong2 rm, rb;
    rm.x = split_reduce(am[a][0], m);
    rm.y = split_reduce(am[a][1], m);
    rb.x = split_reduce(ab[a][0], m);
    rb.y = split_reduce(ab[a][1], m);
    *reinterpret_cast<ulonglong2*>(o) = rm;
    *reinterpret_cast<ulonglong2*>(o + n) = rb;
  }
}

// Schoolbook variant for rings whose modulus has no NTT (the toy presets:
// q2 a power of two, "eval" = coefficient form). One thread per (j, t):
// out[t] = sum_i sum_s db[i][j][s] * sel_i[t - s] (negacyclic), exact mod 2^64.
__global__ void k_first_dim_schoolbook(const u64* __restrict__ db, const u64* __restrict__ sel, u64* __restrict__ out,
                                       int I, int J, int n, DevMod m) {
  long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long)J * n) return;
  int j = (int)(gid / n), t = (int)(gid % n);
  u64 accm = 0, accb = 0;     // wrapping sums (power-of-two q only)
  Acc128 pm{0, 0}, nm{0, 0}, pb{0, 0}, nb{0, 0};  // exact sums (other q)
  const bool pow2 = m.log2q >= 0;
  for (int i = 0; i < I; ++i) {
    const u64* c = db + ((size_t)i * J + j) * n;
    const u64* sm = sel + (size_t)(2 * i) * n;
    const u64* sb = sel + (size_t)(2 * i + 1) * n;
    for (int s = 0; s < n; ++s) {
      int k = t - s;
      bool neg = k < 0;
      if (neg) k += n;
      u64 dv = c[s];
      if (pow2) {
        u64 a = dv * sm[k], b = dv * sb[k];
        accm += neg ? (u64)0 - a : a;
        accb += neg ? (u64)0 - b : b;
      } else if (neg) {
        mac128(nm, dv, sm[k]);
        mac128(nb, dv, sb[k]);
      } else {
        mac128(pm, dv, sm[k]);
        mac128(pb, dv, sb[k]);
      }
    }
  }
  u64 rm, rb;
  if (pow2) {
    rm = accm & (m.q - 1);
    rb = accb & (m.q - 1);
  } else {
    rm = submod(reduce128(pm.hi, pm.lo, m), reduce128(nm.hi, nm.lo, m), m.q);
    rb = submod(reduce128(pb.hi, pb.lo, m), reduce128(nb.hi, nb.lo, m), m.q);
  }
  out[(size_t)(2 * j) * n + t] = rm;
  out[(size_t)(2 * j + 1) * n + t] = rb;
}

int first_dim_variants() { return 3; }
static int jpt_of(int v) { return v == 0 ? 2 : (v == 1 ? 4 : 8); }

bool first_dim_split_ok(int I, int n, u64 q) { return I <= 4096 && q < (1ull << 34) && n % 2 == 0; }

void first_dim_eval(const u64* db, const u64* sel_eval, u64* out_eval, int I, int J, int n, const DevMod& m, bool ntt,
                    cudaStream_t st, uint2* sel_split, int variant) {
  if (ntt && sel_split && first_dim_split_ok(I, n, m.q)) {
    long cnt = (long)I * 2 * n;
    k_split_sel<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(sel_eval, sel_split, cnt);
    VIA_LAUNCHED();
    int jpt = jpt_of(variant);
    while (J % jpt) jpt >>= 1;
    dim3 grid((n + FD_THREADS * FD_TPT - 1) / (FD_THREADS * FD_TPT), J / jpt);
    switch (jpt) {
      case 8: k_first_dim_ntt<8><<<grid, FD_THREADS, 0, st>>>(db, sel_split, out_eval, I, J, n, m); break;
      case 4: k_first_dim_ntt<4><<<grid, FD_THREADS, 0, st>>>(db, sel_split, out_eval, I, J, n, m); break;
      case 2: k_first_dim_ntt<2><<<grid, FD_THREADS, 0, st>>>(db, sel_split, out_eval, I, J, n, m); break;
      default: k_first_dim_ntt<1><<<grid, FD_THREADS, 0, st>>>(db, sel_split, out_eval, I, J, n, m); break;
    }
  } else if (!ntt) {
    long total = (long)J * n;
    k_first_dim_schoolbook<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(db, sel_eval, out_eval, I, J, n, m);
  } else {
    throw CudaError(100, "first_dim: shape outside the split-accumulator bounds (I <= 4096, q2 < 2^34)");
  }
  VIA_LAUNCHED();
}

void first_dim_eval_batch(const u64* db, const u64* sel_eval, u64* out_eval, int nq, int I, int J, int n,
                          const DevMod& m, bool ntt, cudaStream_t st, uint2* sel_split, int variant) {
  if (nq == 1 || !ntt || !first_dim_split_ok(I, n, m.q)) {
    for (int q = 0; q < nq; ++q)
      first_dim_eval(db, sel_eval + (size_t)q * I * 2 * n, out_eval + (size_t)q * J * 2 * n, I, J, n, m, ntt, st,
                     sel_split, variant);
    return;
  }
  long cnt = (long)nq * I * 2 * n;
  k_split_sel<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(sel_eval, sel_split, cnt);
  VIA_LAUNCHED();
  const unsigned gx = (unsigned)((n + FD_THREADS * FD_TPT - 1) / (FD_THREADS * FD_TPT));
  int q0 = 0;
  const int groups8 = nq / 8;
  if (groups8) {
    k_first_dim_multi<8><<<dim3(gx, J, groups8), FD_THREADS, 0, st>>>(db, sel_split, out_eval, I, J, n, q0, m);
    VIA_LAUNCHED();
    q0 += groups8 * 8;
  }
  if (nq - q0 >= 4) {
    k_first_dim_multi<4><<<dim3(gx, J, 1), FD_THREADS, 0, st>>>(db, sel_split, out_eval, I, J, n, q0, m);
    VIA_LAUNCHED();
    q0 += 4;
  }
  for (; q0 < nq; ++q0) {
    k_first_dim_multi<1><<<dim3(gx, J, 1), FD_THREADS, 0, st>>>(db, sel_split, out_eval, I, J, n, q0, m);
    VIA_LAUNCHED();
  }
}

}  // namespace via
