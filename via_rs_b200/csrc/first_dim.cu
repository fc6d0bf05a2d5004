// FirstDim for rings whose q2 has no NTT (crates/via-server/src/first_dim.rs:94-184
// with the identity "eval" form of prim/algebra/ring/ntt_abstraction.rs:130-158):
// every product is a negacyclic schoolbook convolution. The NTT-friendly moduli
// take the tensor-core scan in fd_tc.cu.
#include "first_dim.cuh"

namespace via {

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

void first_dim_schoolbook(const u64* db, const u64* sel, u64* out, int I, int J, int n, const DevMod& m,
                          cudaStream_t st) {
  long total = (long)J * n;
  k_first_dim_schoolbook<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(db, sel, out, I, J, n, m);
  VIA_LAUNCHED();
}

}  // namespace via
