// FirstDim — the database scan (crates/via-server/src/first_dim.rs:94-184).
//
//   c_j = sum_i sel_i (.) db[i][j]   for every column j, mask and body,
//
// computed pointwise in the eval domain at q2. The database is HBM-resident in
// eval form, one u64 per residue, laid out [i][j][t] (t = eval slot), so that a
// warp reads 512 contiguous bytes per (i, j) and each thread streams its column
// group with 16-byte loads. Products are summed exactly in 128 bits and reduced
// once per output residue (sum < I * q2^2 < 2^128).
#include "first_dim.cuh"

namespace via {

constexpr int FD_TPT = 2;  // eval slots per thread (one 16-byte load)
constexpr int FD_THREADS = 128;

template <int JPT>
__global__ void __launch_bounds__(FD_THREADS) k_first_dim_ntt(const u64* __restrict__ db, const u64* __restrict__ sel,
                                                              u64* __restrict__ out, int I, int J, int n, DevMod m) {
  const int t = (blockIdx.x * FD_THREADS + threadIdx.x) * FD_TPT;
  const int j0 = blockIdx.y * JPT;
  if (t >= n) return;
  Acc128 am[JPT][FD_TPT], ab[JPT][FD_TPT];
#pragma unroll
  for (int jj = 0; jj < JPT; ++jj)
#pragma unroll
    for (int k = 0; k < FD_TPT; ++k) am[jj][k] = ab[jj][k] = Acc128{0, 0};
  const size_t row_stride = (size_t)J * n;
  const u64* dbp = db + (size_t)j0 * n + t;
  for (int i = 0; i < I; ++i) {
    const ulonglong2 sm = *reinterpret_cast<const ulonglong2*>(sel + (size_t)(2 * i) * n + t);
    const ulonglong2 sb = *reinterpret_cast<const ulonglong2*>(sel + (size_t)(2 * i + 1) * n + t);
    ulonglong2 d[JPT];
#pragma unroll
    for (int jj = 0; jj < JPT; ++jj) d[jj] = __ldcs(reinterpret_cast<const ulonglong2*>(dbp + (size_t)jj * n));
#pragma unroll
    for (int jj = 0; jj < JPT; ++jj) {
      mac128(am[jj][0], d[jj].x, sm.x);
      mac128(am[jj][1], d[jj].y, sm.y);
      mac128(ab[jj][0], d[jj].x, sb.x);
      mac128(ab[jj][1], d[jj].y, sb.y);
    }
    dbp += row_stride;
  }
#pragma unroll
  for (int jj = 0; jj < JPT; ++jj) {
    u64* o = out + (size_t)(2 * (j0 + jj)) * n + t;
    ulonglong2 rm, rb;
    rm.x = reduce128(am[jj][0].hi, am[jj][0].lo, m);
    rm.y = reduce128(am[jj][1].hi, am[jj][1].lo, m);
    rb.x = reduce128(ab[jj][0].hi, ab[jj][0].lo, m);
    rb.y = reduce128(ab[jj][1].hi, ab[jj][1].lo, m);
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

void first_dim_eval(const u64* db, const u64* sel_eval, u64* out_eval, int I, int J, int n, const DevMod& m,
                    bool ntt, cudaStream_t st) {
  if (ntt) {
    constexpr int JPT = 8;
    if (J % JPT != 0 || n % (FD_THREADS * FD_TPT) != 0) {
      // Small shapes: one column per thread group.
      dim3 grid((n + FD_THREADS * FD_TPT - 1) / (FD_THREADS * FD_TPT), J);
      k_first_dim_ntt<1><<<grid, FD_THREADS, 0, st>>>(db, sel_eval, out_eval, I, J, n, m);
    } else {
      dim3 grid(n / (FD_THREADS * FD_TPT), J / JPT);
      k_first_dim_ntt<JPT><<<grid, FD_THREADS, 0, st>>>(db, sel_eval, out_eval, I, J, n, m);
    }
  } else {
    long total = (long)J * n;
    k_first_dim_schoolbook<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(db, sel_eval, out_eval, I, J, n, m);
  }
  VIA_LAUNCHED();
}

}  // namespace via
