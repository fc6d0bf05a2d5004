// Batched negacyclic NTT kernels (shared-memory staged, radix-2, Shoup twiddles).
#include <cstring>

#include "ntt.cuh"

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
  std::vector<u64> host(4 * (size_t)nmax);
  for (int k = 0; k < nmax; ++k) {
    u64 w = h_pow(psi, (u64)bitrev(k, logn), q);
    u64 wi = h_pow(ipsi, (u64)bitrev(k, logn), q);
    host[k] = w;
    host[nmax + k] = (u64)(((u128)w << 64) / q);
    host[2 * nmax + k] = wi;
    host[3 * nmax + k] = (u64)(((u128)wi << 64) / q);
  }
  VIA_CUDA(cudaMalloc(&h.buf, host.size() * 8));
  VIA_CUDA(cudaMemcpy(h.buf, host.data(), host.size() * 8, cudaMemcpyHostToDevice));
  h.dev.q = q;
  h.dev.nmax = nmax;
  h.dev.psi = h.buf;
  h.dev.psi_sh = h.buf + nmax;
  h.dev.ipsi = h.buf + 2 * nmax;
  h.dev.ipsi_sh = h.buf + 3 * nmax;
  for (int l = 0; l <= NTT_MAX_LOGN; ++l) {
    u64 ninv = h_pow((u64)1 << l, q - 2, q);
    h.dev.ninv[l] = ninv;
    h.dev.ninv_sh[l] = (u64)(((u128)ninv << 64) / q);
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

// One CTA transforms a tile of `tile` coefficients (tile/n whole segments).
template <bool INV>
__global__ void __launch_bounds__(NTT_THREADS) k_ntt(u64* __restrict__ data, int logn, int nl, long segments,
                                                     int tile, NttTable t0, NttTable t1) {
  extern __shared__ u64 sm[];
  const int n = 1 << logn;
  const int spt = tile >> logn;  // segments per tile
  const long seg0 = (long)blockIdx.x * spt;
  const int nseg = (int)min((long)spt, segments - seg0);
  const int count = nseg << logn;
  u64* g = data + (seg0 << logn);
  for (int i = threadIdx.x; i < count; i += NTT_THREADS) sm[i] = g[i];
  __syncthreads();
  const int half = n >> 1;
  const int nbf = count >> 1;  // butterflies per stage
  if (!INV) {
    for (int len = half, m = 1; len >= 1; len >>= 1, m <<= 1) {
      for (int b = threadIdx.x; b < nbf; b += NTT_THREADS) {
        int sl = b >> (logn - 1), bb = b & (half - 1);
        int grp = bb / len, j = bb - grp * len;
        int i0 = (sl << logn) + grp * 2 * len + j, i1 = i0 + len;
        const NttTable& T = (nl == 2 && ((seg0 + sl) & 1)) ? t1 : t0;
        u64 q = T.q;
        u64 u = sm[i0];
        u64 v = mul_shoup(sm[i1], T.psi[m + grp], T.psi_sh[m + grp], q);
        sm[i0] = addmod(u, v, q);
        sm[i1] = submod(u, v, q);
      }
      __syncthreads();
    }
  } else {
    for (int len = 1, m = half; len < n; len <<= 1, m >>= 1) {
      for (int b = threadIdx.x; b < nbf; b += NTT_THREADS) {
        int sl = b >> (logn - 1), bb = b & (half - 1);
        int grp = bb / len, j = bb - grp * len;
        int i0 = (sl << logn) + grp * 2 * len + j, i1 = i0 + len;
        const NttTable& T = (nl == 2 && ((seg0 + sl) & 1)) ? t1 : t0;
        u64 q = T.q;
        u64 u = sm[i0], v = sm[i1];
        sm[i0] = addmod(u, v, q);
        sm[i1] = mul_shoup(submod(u, v, q), T.ipsi[m + grp], T.ipsi_sh[m + grp], q);
      }
      __syncthreads();
    }
    for (int i = threadIdx.x; i < count; i += NTT_THREADS) {
      int sl = i >> logn;
      const NttTable& T = (nl == 2 && ((seg0 + sl) & 1)) ? t1 : t0;
      sm[i] = mul_shoup(sm[i], T.ninv[logn], T.ninv_sh[logn], T.q);
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < count; i += NTT_THREADS) g[i] = sm[i];
}

template <bool INV>
static void launch(u64* data, int n, int nl, long segments, const NttTable& t0, const NttTable& t1,
                   cudaStream_t st) {
  if (segments <= 0) return;
  int logn = __builtin_ctz((unsigned)n);
  if (n < 2 || (n & (n - 1)) || logn > NTT_MAX_LOGN) throw CudaError(100, "ntt: bad degree");
  int tile = n > 2048 ? n : 2048;
  long spt = tile / n;
  long blocks = (segments + spt - 1) / spt;
  size_t smem = (size_t)tile * 8;
  if (smem > 48 * 1024) VIA_CUDA(cudaFuncSetAttribute(k_ntt<INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_ntt<INV><<<(unsigned)blocks, NTT_THREADS, smem, st>>>(data, logn, nl, segments, tile, t0, t1);
  VIA_LAUNCHED();
}

void ntt_forward(u64* data, int n, int nl, long segments, const NttTable& t0, const NttTable& t1, cudaStream_t st) {
  launch<false>(data, n, nl, segments, t0, t1, st);
}
void ntt_inverse(u64* data, int n, int nl, long segments, const NttTable& t0, const NttTable& t1, cudaStream_t st) {
  launch<true>(data, n, nl, segments, t0, t1, st);
}

}  // namespace via
