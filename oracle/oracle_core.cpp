// CPU oracle, part 1: Keccak/SHAKE-256 PRG, samplers, moduli, rings, NTT.
// Test infrastructure only (see via_oracle.hpp).
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>

#include "via_oracle.hpp"

namespace vo {

// ===========================================================================
// Keccak-f[1600] and SHAKE-256, written from FIPS 202 (sections 3.2, 5, 6.2).
// The SHAKE-256 XOF is the third-party `sha3 0.10.9` dependency behind
// prim/sampling/prg.rs:117-128; this is a restatement of the published standard.
// ===========================================================================
namespace {
struct KeccakConsts {
  u64 rc[24];
  int rot[25];
  KeccakConsts() {
    // Round constants from the degree-8 LFSR rc(t) (FIPS 202 Algorithm 5).
    auto rc_bit = [](int t) {
      if (t % 255 == 0) return 1;
      u32 R = 1;  // R = 10000000 as bits r0..r7 (r0 = LSB here)
      for (int i = 1; i <= t % 255; ++i) {
        u32 r8 = (R >> 7) & 1;  // bit shifted out
        R = (R << 1) & 0x1FF;   // prepend 0
        // R[0] ^= R[8]; R[4] ^= R[8]; R[5] ^= R[8]; R[6] ^= R[8]
        if (r8) R ^= (1u << 0) | (1u << 4) | (1u << 5) | (1u << 6);
        R &= 0xFF;
      }
      return (int)(R & 1);
    };
    for (int ir = 0; ir < 24; ++ir) {
      u64 c = 0;
      for (int j = 0; j <= 6; ++j)
        if (rc_bit(j + 7 * ir)) c |= (u64)1 << ((1 << j) - 1);
      rc[ir] = c;
    }
    // Rotation offsets (FIPS 202 Algorithm 2 rho).
    for (int i = 0; i < 25; ++i) rot[i] = 0;
    int x = 1, y = 0;
    for (int t = 0; t < 24; ++t) {
      rot[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
      int nx = y, ny = (2 * x + 3 * y) % 5;
      x = nx;
      y = ny;
    }
  }
};
const KeccakConsts& kc() {
  static KeccakConsts k;
  return k;
}
inline u64 rotl(u64 v, int r) { return r == 0 ? v : (v << r) | (v >> (64 - r)); }

void keccak_f(u64 A[25]) {
  const auto& K = kc();
  for (int ir = 0; ir < 24; ++ir) {
    u64 C[5], D[5], B[25];
    for (int x = 0; x < 5; ++x) C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
    for (int x = 0; x < 5; ++x) D[x] = C[(x + 4) % 5] ^ rotl(C[(x + 1) % 5], 1);
    for (int i = 0; i < 25; ++i) A[i] ^= D[i % 5];
    // rho + pi: B[y, 2x+3y] = rot(A[x,y])
    for (int x = 0; x < 5; ++x)
      for (int y = 0; y < 5; ++y) B[y + 5 * ((2 * x + 3 * y) % 5)] = rotl(A[x + 5 * y], K.rot[x + 5 * y]);
    // chi
    for (int y = 0; y < 5; ++y)
      for (int x = 0; x < 5; ++x)
        A[x + 5 * y] = B[x + 5 * y] ^ ((~B[(x + 1) % 5 + 5 * y]) & B[(x + 2) % 5 + 5 * y]);
    // iota
    A[0] ^= K.rc[ir];
  }
}
}  // namespace

void shake256(const u8* in, size_t inlen, u8* out, size_t outlen) {
  const size_t rate = 136;
  u64 A[25] = {0};
  auto absorb_block = [&](const u8* blk) {
    for (size_t i = 0; i < rate / 8; ++i) {
      u64 w = 0;
      for (int b = 0; b < 8; ++b) w |= (u64)blk[8 * i + b] << (8 * b);
      A[i] ^= w;
    }
    keccak_f(A);
  };
  size_t off = 0;
  while (inlen - off >= rate) {
    absorb_block(in + off);
    off += rate;
  }
  u8 last[136];
  std::memset(last, 0, rate);
  std::memcpy(last, in + off, inlen - off);
  last[inlen - off] ^= 0x1F;  // SHAKE domain bits 1111 + first pad bit
  last[rate - 1] ^= 0x80;
  absorb_block(last);
  size_t produced = 0;
  while (true) {
    for (size_t i = 0; i < rate && produced < outlen; ++i, ++produced)
      out[produced] = (u8)(A[i / 8] >> (8 * (i % 8)));
    if (produced >= outlen) break;
    keccak_f(A);
  }
}

Prg::Prg(const void* s, size_t len) {
  if (len > 64) throw OracleError(ERR_INVALID, "seed longer than 64 bytes");
  std::memset(seed, 0, sizeof seed);
  std::memcpy(seed, s, len);
  seed_len = len;
}

void Prg::refill() {
  u8 msg[72];
  std::memcpy(msg, seed, seed_len);
  for (int b = 0; b < 8; ++b) msg[seed_len + b] = (u8)(counter >> (8 * b));
  shake256(msg, seed_len + 8, buf, 136);
  counter += 1;
  pos = 0;
}

void Prg::fill(u8* out, size_t n) {
  size_t w = 0;
  while (w < n) {
    if (pos >= 136) refill();
    size_t take = std::min(n - w, (size_t)136 - pos);
    std::memcpy(out + w, buf + pos, take);
    pos += take;
    w += take;
  }
}

u64 Prg::uniform_below(u64 bound) {
  if (bound == 0) throw OracleError(ERR_INVALID, "bound must be positive");
  if (bound == 1) return 0;
  int bits = 64 - __builtin_clzll(bound);
  size_t nbytes = (size_t)(bits + 7) / 8;
  u64 mask = bits == 64 ? ~(u64)0 : (((u64)1 << bits) - 1);
  u8 b[8] = {0};
  for (;;) {
    fill(b, nbytes);
    u64 v = 0;
    for (int i = 0; i < 8; ++i) v |= (u64)b[i] << (8 * i);
    v &= mask;
    if (v < bound) return v;
  }
}

void sample_into(const Dist& d, Prg& prg, i64* out, size_t n) {
  if (d.kind == 0) {
    for (size_t i = 0; i < n; ++i) {
      u64 r = prg.uniform_below(3);
      out[i] = r == 0 ? 0 : (r == 1 ? 1 : -1);
    }
  } else {
    u64 range = 2 * (u64)d.bound + 1;
    for (size_t i = 0; i < n; ++i) out[i] = (i64)prg.uniform_below(range) - (i64)d.bound;
  }
}

// ===========================================================================
// Modulus — prim/algebra/zq/{modulus,reduce}.rs.
// ===========================================================================
static u128 umul128_hi(u128 x, u128 mu) {
  u128 xl = (u64)x, xh = x >> 64, ml = (u64)mu, mh = mu >> 64;
  u128 p00 = xl * ml, p01 = xl * mh, p10 = xh * ml, p11 = xh * mh;
  u128 carry = ((p00 >> 64) + (u64)p01 + (u64)p10) >> 64;
  return p11 + (p01 >> 64) + (p10 >> 64) + carry;
}

Mod::Mod(u64 q_) : q(q_) {
  if (q < 2) throw OracleError(ERR_INVALID, "modulus must be >= 2");
  if ((q & (q - 1)) == 0) {
    log2q = __builtin_ctzll(q);
  } else {
    if (q >= ((u64)1 << 63)) throw OracleError(ERR_INVALID, "modulus must be < 2^63");
    u128 qq = q;
    u128 approx = ~(u128)0 / qq;
    u128 r = (~(u128)0 % qq + 1) % qq;
    mu = r == 0 ? approx + 1 : approx;
  }
}

u64 Mod::reduce(u128 x) const {
  if (log2q >= 0) return (u64)(x & (((u128)1 << log2q) - 1));
  u128 qh = umul128_hi(x, mu);
  u64 r = (u64)(x - qh * q);
  return r >= q ? r - q : r;
}

u64 Mod::reduce_i64(i64 x) const {
  u64 mag = x < 0 ? (u64)0 - (u64)x : (u64)x;
  u64 r = reduce(mag);
  return x < 0 ? neg(r) : r;
}

// ===========================================================================
// Negacyclic NTT over Z_q (q prime, 2n | q-1). The evaluation layout is internal
// to this oracle: only coefficient-form values are ever compared.
// ===========================================================================
struct NttTable {
  u64 q = 0;
  int n = 0;
  Mod m;
  std::vector<u64> psi_rev;      // psi^{bitrev(i)}
  std::vector<u64> psi_inv_rev;  // psi^{-bitrev(i)}
  u64 n_inv = 0;
};

static u64 powmod(const Mod& m, u64 b, u64 e) {
  u64 r = 1 % m.q;
  b %= m.q;
  while (e) {
    if (e & 1) r = m.mul(r, b);
    b = m.mul(b, b);
    e >>= 1;
  }
  return r;
}

static bool is_prime_u64(u64 n) {
  if (n < 2) return false;
  for (u64 p : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
    if (n % p == 0) return n == p;
  }
  u64 d = n - 1;
  int s = 0;
  while ((d & 1) == 0) {
    d >>= 1;
    ++s;
  }
  Mod m(n);
  for (u64 a : {2ull, 3ull, 5ull, 7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull, 37ull}) {
    u64 x = powmod(m, a, d);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int r = 1; r < s; ++r) {
      x = m.mul(x, x);
      if (x == n - 1) {
        comp = false;
        break;
      }
    }
    if (comp) return false;
  }
  return true;
}

static int bitrev(int x, int logn) {
  int r = 0;
  for (int i = 0; i < logn; ++i) r |= ((x >> i) & 1) << (logn - 1 - i);
  return r;
}

static const NttTable* get_ntt(u64 q, int n) {
  static std::mutex mu;
  static std::map<std::pair<u64, int>, NttTable*> cache;
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_pair(q, n);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  NttTable* t = nullptr;
  if (n >= 2 && (q & (q - 1)) != 0 && (q - 1) % (2 * (u64)n) == 0 && is_prime_u64(q)) {
    t = new NttTable();
    t->q = q;
    t->n = n;
    t->m = Mod(q);
    // Find a primitive 2n-th root of unity: g^((q-1)/2n) with psi^n = -1.
    u64 psi = 0;
    for (u64 g = 2; g < q; ++g) {
      u64 cand = powmod(t->m, g, (q - 1) / (2 * (u64)n));
      if (powmod(t->m, cand, (u64)n) == q - 1) {
        psi = cand;
        break;
      }
    }
    int logn = __builtin_ctz((unsigned)n);
    t->psi_rev.resize(n);
    t->psi_inv_rev.resize(n);
    u64 psi_inv = powmod(t->m, psi, q - 2);
    for (int i = 0; i < n; ++i) {
      t->psi_rev[i] = powmod(t->m, psi, (u64)bitrev(i, logn));
      t->psi_inv_rev[i] = powmod(t->m, psi_inv, (u64)bitrev(i, logn));
    }
    t->n_inv = powmod(t->m, (u64)n, q - 2);
  }
  cache[key] = t;
  return t;
}

static void ntt_fwd(const NttTable& T, u64* a) {
  const Mod& m = T.m;
  int n = T.n;
  int k = 1;
  for (int len = n / 2; len >= 1; len >>= 1) {
    for (int start = 0; start < n; start += 2 * len) {
      u64 w = T.psi_rev[k++];
      for (int j = start; j < start + len; ++j) {
        u64 u = a[j], v = m.mul(a[j + len], w);
        a[j] = m.add(u, v);
        a[j + len] = m.sub(u, v);
      }
    }
  }
}

static void ntt_inv(const NttTable& T, u64* a) {
  const Mod& m = T.m;
  int n = T.n;
  int k = n - 1;
  for (int len = 1; len < n; len <<= 1) {
    for (int start = n - 2 * len; start >= 0; start -= 2 * len) {
      u64 w = T.psi_inv_rev[k--];
      for (int j = start; j < start + len; ++j) {
        u64 u = a[j], v = a[j + len];
        a[j] = m.add(u, v);
        a[j + len] = m.mul(m.sub(u, v), w);
      }
    }
  }
  for (int j = 0; j < n; ++j) a[j] = m.mul(a[j], T.n_inv);
}

// ===========================================================================
// Ring — prim/algebra/ring/{element,rns_element,ops,reshape}.rs.
// ===========================================================================
static u64 mod_inverse(u64 a, u64 m) {
  i128 t = 0, nt = 1, r = m, nr = a % m;
  while (nr != 0) {
    i128 qq = r / nr;
    i128 tmp = t - qq * nt;
    t = nt;
    nt = tmp;
    tmp = r - qq * nr;
    r = nr;
    nr = tmp;
  }
  if (r != 1) return 0;
  if (t < 0) t += m;
  return (u64)t;
}

Ring Ring::single(int n, u64 q) {
  Ring R;
  R.n = n;
  R.nl = 1;
  R.m[0] = Mod(q);
  R.ntt[0] = get_ntt(q, n);
  return R;
}

Ring Ring::rns(int n, u64 q0, u64 q1) {
  Ring R;
  R.n = n;
  R.nl = 2;
  R.m[0] = Mod(q0);
  R.m[1] = Mod(q1);
  R.q0inv_mod_q1 = mod_inverse(q0 % q1, q1);
  if (R.q0inv_mod_q1 == 0) throw OracleError(ERR_INVALID, "RNS primes not coprime");
  const NttTable* t0 = get_ntt(q0, n);
  const NttTable* t1 = get_ntt(q1, n);
  if (t0 && t1) {
    R.ntt[0] = t0;
    R.ntt[1] = t1;
  }
  return R;
}

Ring Ring::with_n(int n2) const {
  return nl == 1 ? Ring::single(n2, m[0].q) : Ring::rns(n2, m[0].q, m[1].q);
}

Poly Ring::add(const Poly& a, const Poly& b) const {
  Poly r(size());
  for (int l = 0; l < nl; ++l)
    for (int i = 0; i < n; ++i) r[l * n + i] = m[l].add(a[l * n + i], b[l * n + i]);
  return r;
}
Poly Ring::sub(const Poly& a, const Poly& b) const {
  Poly r(size());
  for (int l = 0; l < nl; ++l)
    for (int i = 0; i < n; ++i) r[l * n + i] = m[l].sub(a[l * n + i], b[l * n + i]);
  return r;
}
Poly Ring::neg(const Poly& a) const {
  Poly r(size());
  for (int l = 0; l < nl; ++l)
    for (int i = 0; i < n; ++i) r[l * n + i] = m[l].neg(a[l * n + i]);
  return r;
}
void Ring::add_inplace(Poly& a, const Poly& b) const {
  for (int l = 0; l < nl; ++l)
    for (int i = 0; i < n; ++i) a[l * n + i] = m[l].add(a[l * n + i], b[l * n + i]);
}
void Ring::sub_inplace(Poly& a, const Poly& b) const {
  for (int l = 0; l < nl; ++l)
    for (int i = 0; i < n; ++i) a[l * n + i] = m[l].sub(a[l * n + i], b[l * n + i]);
}

// Schoolbook negacyclic product — prim/algebra/ring/ops.rs:65-110. For a power
// of two modulus the product is taken with wrapping u64 arithmetic (exact
// modulo 2^64, hence modulo q); otherwise the signed sums are kept in i128.
static void schoolbook(const Mod& m, int n, const u64* a, const u64* b, u64* out) {
  if (m.log2q >= 0) {
    std::vector<u64> acc(n, 0);
    for (int i = 0; i < n; ++i) {
      if (a[i] == 0) continue;
      for (int j = 0; j < n; ++j) {
        u64 p = a[i] * b[j];
        int k = i + j;
        if (k < n)
          acc[k] += p;
        else
          acc[k - n] -= p;
      }
    }
    for (int k = 0; k < n; ++k) out[k] = m.reduce(acc[k]);
  } else {
    std::vector<u64> acc(n, 0);
    for (int k = 0; k < n; ++k) {
      // Sum positive and negative parts separately as residues.
      u128 pos = 0, neg = 0;
      u64 pos_r = 0, neg_r = 0;
      for (int i = 0; i < n; ++i) {
        int j = k - i;
        u128 p;
        if (j >= 0) {
          p = (u128)a[i] * b[j];
          pos += p;
          if (pos >> 120) {
            pos_r = m.add(pos_r, m.reduce(pos));
            pos = 0;
          }
        } else {
          p = (u128)a[i] * b[j + n];
          neg += p;
          if (neg >> 120) {
            neg_r = m.add(neg_r, m.reduce(neg));
            neg = 0;
          }
        }
      }
      pos_r = m.add(pos_r, m.reduce(pos));
      neg_r = m.add(neg_r, m.reduce(neg));
      out[k] = m.sub(pos_r, neg_r);
    }
  }
}

Poly Ring::mul(const Poly& a, const Poly& b) const {
  if (eval_is_ntt()) return from_eval(mul_eval(to_eval(a), to_eval(b)));
  Poly r(size());
  for (int l = 0; l < nl; ++l) schoolbook(m[l], n, &a[l * n], &b[l * n], &r[l * n]);
  return r;
}

Poly Ring::to_eval(const Poly& a) const {
  if (!eval_is_ntt()) return a;
  Poly r = a;
  for (int l = 0; l < nl; ++l) ntt_fwd(*ntt[l], &r[l * n]);
  return r;
}
Poly Ring::from_eval(const Poly& a) const {
  if (!eval_is_ntt()) return a;
  Poly r = a;
  for (int l = 0; l < nl; ++l) ntt_inv(*ntt[l], &r[l * n]);
  return r;
}
Poly Ring::mul_eval(const Poly& a, const Poly& b) const {
  Poly r(size());
  if (eval_is_ntt()) {
    for (int l = 0; l < nl; ++l)
      for (int i = 0; i < n; ++i) r[l * n + i] = m[l].mul(a[l * n + i], b[l * n + i]);
  } else {
    for (int l = 0; l < nl; ++l) schoolbook(m[l], n, &a[l * n], &b[l * n], &r[l * n]);
  }
  return r;
}
void Ring::mac_eval(Poly& acc, const Poly& a, const Poly& b) const {
  if (eval_is_ntt()) {
    for (int l = 0; l < nl; ++l)
      for (int i = 0; i < n; ++i) acc[l * n + i] = m[l].add(acc[l * n + i], m[l].mul(a[l * n + i], b[l * n + i]));
  } else {
    add_inplace(acc, mul_eval(a, b));
  }
}

Poly Ring::from_u128(const std::vector<u128>& v) const {
  Poly r(size());
  for (int l = 0; l < nl; ++l)
    for (int i = 0; i < n; ++i) r[l * n + i] = m[l].reduce(v[i]);
  return r;
}

// prim/algebra/rns/basis.rs reconstruct: a0 + q0 * ((a1 - a0) * q0^{-1} mod q1).
static inline u128 crt2(const Ring& R, u64 a0, u64 a1) {
  u64 a0m = R.m[1].reduce(a0);
  u64 diff = R.m[1].sub(a1, a0m);
  u64 t = R.m[1].mul(diff, R.q0inv_mod_q1);
  return (u128)a0 + (u128)R.m[0].q * t;
}

std::vector<u128> Ring::to_u128(const Poly& a) const {
  std::vector<u128> r(n);
  for (int i = 0; i < n; ++i) r[i] = nl == 1 ? (u128)a[i] : crt2(*this, a[i], a[n + i]);
  return r;
}

std::vector<i128> Ring::centered(const Poly& a) const {
  std::vector<i128> r(n);
  u128 Qv = Q(), half = Qv / 2;
  for (int i = 0; i < n; ++i) {
    u128 v = nl == 1 ? (u128)a[i] : crt2(*this, a[i], a[n + i]);
    r[i] = v <= half ? (i128)v : (i128)v - (i128)Qv;
  }
  return r;
}

Poly Ring::from_centered_i64(const i64* s) const {
  Poly r(size());
  for (int l = 0; l < nl; ++l)
    for (int i = 0; i < n; ++i) r[l * n + i] = m[l].reduce_i64(s[i]);
  return r;
}

Poly Ring::from_centered_i128(const std::vector<i128>& s) const {
  Poly r(size());
  for (int l = 0; l < nl; ++l)
    for (int i = 0; i < n; ++i) {
      if (nl == 1) {
        r[i] = m[0].reduce_i64((i64)s[i]);
      } else {
        u128 mag = s[i] < 0 ? (u128)(-s[i]) : (u128)s[i];
        u64 v = m[l].reduce(mag);
        r[l * n + i] = s[i] < 0 ? m[l].neg(v) : v;
      }
    }
  return r;
}

Poly Ring::random_uniform(Prg& prg) const {
  Poly r(size());
  for (int i = 0; i < n; ++i)
    for (int l = 0; l < nl; ++l) r[l * n + i] = prg.uniform_below(m[l].q);
  return r;
}

// prim/algebra/ring/ops.rs:147-180 rotate_slice.
Poly Ring::mul_x_pow(const Poly& a, size_t k) const {
  Poly r(size());
  size_t keff = k % (2 * (size_t)n);
  size_t kred = keff % n;
  bool neg_global = keff >= (size_t)n;
  for (int l = 0; l < nl; ++l)
    for (int i = 0; i < n; ++i) {
      bool wrapped = (size_t)i + kred >= (size_t)n;
      size_t out = wrapped ? i + kred - n : i + kred;
      u64 v = a[l * n + i];
      r[l * n + out] = (wrapped ^ neg_global) ? m[l].neg(v) : v;
    }
  return r;
}

Poly Ring::scalar_const(u128 c) const {
  std::vector<u128> v(n, 0);
  v[0] = c;
  return from_u128(v);
}

// prim/algebra/ring/reshape.rs:58 embed_at_slice: coeff i -> position d*i + slot.
Poly embed_at(const Ring& src, const Poly& a, int n_large, int slot) {
  int d = n_large / src.n;
  Poly r((size_t)src.nl * n_large, 0);
  for (int l = 0; l < src.nl; ++l)
    for (int i = 0; i < src.n; ++i) r[(size_t)l * n_large + (size_t)d * i + slot] = a[(size_t)l * src.n + i];
  return r;
}

// prim/algebra/ring/reshape.rs:93 project_at_slice: dst[i] = src[d*i + slot].
Poly project_at(const Ring& src, const Poly& a, int n_small, int slot) {
  int d = src.n / n_small;
  Poly r((size_t)src.nl * n_small);
  for (int l = 0; l < src.nl; ++l)
    for (int i = 0; i < n_small; ++i) r[(size_t)l * n_small + i] = a[(size_t)l * src.n + (size_t)d * i + slot];
  return r;
}

}  // namespace vo
