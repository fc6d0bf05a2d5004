// CPU oracle, part 2: gadget, encryption, gates, switching, conversion, client,
// server. Test infrastructure only (see via_oracle.hpp).
#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>

#include "via_oracle.hpp"

namespace vo {

// ===========================================================================
// Wide arithmetic — prim/algebra/wide.rs:145-153 round_mul_div_u128:
// floor((num * scale + floor(divisor/2)) / divisor) with a 256-bit intermediate.
// ===========================================================================
namespace {
struct U256 {
  u64 w[4];
};
U256 mul_u128(u128 a, u128 b) {
  u64 al = (u64)a, ah = (u64)(a >> 64), bl = (u64)b, bh = (u64)(b >> 64);
  u128 p00 = (u128)al * bl, p01 = (u128)al * bh, p10 = (u128)ah * bl, p11 = (u128)ah * bh;
  U256 r;
  r.w[0] = (u64)p00;
  u128 mid = (p00 >> 64) + (u64)p01 + (u64)p10;
  r.w[1] = (u64)mid;
  u128 mid2 = (mid >> 64) + (p01 >> 64) + (p10 >> 64) + (u64)p11;
  r.w[2] = (u64)mid2;
  r.w[3] = (u64)((mid2 >> 64) + (p11 >> 64));
  return r;
}
void add_u128(U256& x, u128 v) {
  u128 s = (u128)x.w[0] + (u64)v;
  x.w[0] = (u64)s;
  s = (s >> 64) + x.w[1] + (u64)(v >> 64);
  x.w[1] = (u64)s;
  s = (s >> 64) + x.w[2];
  x.w[2] = (u64)s;
  x.w[3] += (u64)(s >> 64);
}
void sub_u256(U256& x, const U256& y) {
  u64 borrow = 0;
  for (int i = 0; i < 4; ++i) {
    u128 d = (u128)x.w[i] - y.w[i] - borrow;
    x.w[i] = (u64)d;
    borrow = (u64)(d >> 64) ? 1 : 0;
  }
}
}  // namespace

u128 round_mul_div_u128(u128 num_abs, u128 scale, u128 divisor) {
  if (divisor == 0) throw OracleError(ERR_INVALID, "divisor must be nonzero");
  U256 p = mul_u128(num_abs, scale);
  add_u128(p, divisor / 2);
  if (p.w[2] == 0 && p.w[3] == 0) {
    u128 lo = ((u128)p.w[1] << 64) | p.w[0];
    return lo / divisor;
  }
  // Estimate the quotient in extended precision, then correct it exactly with
  // the (small) signed remainder.
  long double pv = std::ldexp((long double)p.w[3], 192) + std::ldexp((long double)p.w[2], 128) +
                   std::ldexp((long double)p.w[1], 64) + (long double)p.w[0];
  long double qd = pv / (long double)divisor;
  u128 q_est = (u128)qd;
  U256 qd256 = mul_u128(q_est, divisor);
  U256 r = p;
  sub_u256(r, qd256);
  i128 rem = (i128)(((u128)r.w[1] << 64) | r.w[0]);  // |rem| << 2^127
  i128 dv = (i128)divisor;
  i128 adj = rem / dv;
  i128 rr = rem % dv;
  if (rr < 0) adj -= 1;
  return (u128)((i128)q_est + adj);
}

// ===========================================================================
// Gadget — prim/encryption/gadget.rs:73-190.
// ===========================================================================
std::vector<u128> gadget_vector_values(u128 Q, u64 base, int L) {
  std::vector<u128> out(L);
  u128 div = 1;
  for (int i = 0; i < L; ++i) {
    div *= base;
    out[i] = (Q + div / 2) / div;
  }
  return out;
}

void gadget_scale_into(const Ring& R, const Poly& x, u64 base, int L, std::vector<i128>& scratch) {
  u128 Q = R.Q();
  u128 bl = 1;
  for (int i = 0; i < L; ++i) bl *= base;
  std::vector<i128> c = R.centered(x);
  scratch.resize(R.n);
  for (int i = 0; i < R.n; ++i) {
    u128 a = c[i] < 0 ? (u128)(-c[i]) : (u128)c[i];
    u128 v = round_mul_div_u128(a, bl, Q);
    scratch[i] = c[i] >= 0 ? (i128)v : -(i128)v;
  }
}

void gadget_extract_lsb_into(u64 base, std::vector<i128>& scratch, std::vector<i64>& out) {
  i128 B = base, half = B / 2;
  out.resize(scratch.size());
  for (size_t i = 0; i < scratch.size(); ++i) {
    i128 v = scratch[i];
    i128 d = v % B;
    if (d < 0) d += B;  // rem_euclid
    if (d > half) d -= B;
    out[i] = (i64)d;
    scratch[i] = (v - d) / B;
  }
}

Rlwe gadget_product(const Ring& R, const RlevEval& key, const Poly& x, u64 base) {
  int L = (int)key.mask.size();
  std::vector<i128> scratch;
  gadget_scale_into(R, x, base, L, scratch);
  std::vector<i64> digits;
  Poly acc_m = R.zero(), acc_b = R.zero();
  for (int k = 0; k < L; ++k) {
    gadget_extract_lsb_into(base, scratch, digits);
    Poly de = R.to_eval(R.from_centered_i64(digits.data()));
    R.mac_eval(acc_m, de, key.mask[L - 1 - k]);
    R.mac_eval(acc_b, de, key.body[L - 1 - k]);
  }
  return Rlwe{R.from_eval(acc_m), R.from_eval(acc_b)};
}

RlevEval rlev_to_eval(const Ring& R, const Rlev& k) {
  RlevEval e;
  for (auto& s : k) {
    e.mask.push_back(R.to_eval(s.mask));
    e.body.push_back(R.to_eval(s.body));
  }
  return e;
}
RgswEval rgsw_to_eval(const Ring& R, const Rgsw& g) { return RgswEval{rlev_to_eval(R, g.neg_s_m), rlev_to_eval(R, g.m)}; }

Rlwe gadget_product_coeff(const Ring& R, const Rlev& key, const Poly& x, u64 base) {
  return gadget_product(R, rlev_to_eval(R, key), x, base);
}

// prim/encryption/keyswitch.rs:99-102.
Rlwe key_switch(const Ring& R, const RlevEval& key, const Rlwe& ct, u64 base) {
  Rlwe p = gadget_product(R, key, ct.mask, base);
  return Rlwe{R.neg(p.mask), R.sub(ct.body, p.body)};
}

// prim/encryption/rgsw.rs:108-121.
Rlwe external_product(const Ring& R, const RgswEval& g, const Rlwe& ct, u64 b1, u64 b2) {
  Rlwe a = gadget_product(R, g.neg_s_m, ct.mask, b1);
  Rlwe b = gadget_product(R, g.m, ct.body, b2);
  return rlwe_add(R, a, b);
}

Rlwe rlwe_add(const Ring& R, const Rlwe& a, const Rlwe& b) { return Rlwe{R.add(a.mask, b.mask), R.add(a.body, b.body)}; }
Rlwe rlwe_sub(const Ring& R, const Rlwe& a, const Rlwe& b) { return Rlwe{R.sub(a.mask, b.mask), R.sub(a.body, b.body)}; }
Rlwe rlwe_neg(const Ring& R, const Rlwe& a) { return Rlwe{R.neg(a.mask), R.neg(a.body)}; }

// ===========================================================================
// Secret-key side — prim/encryption/rlwe.rs, rlev.rs, rgsw.rs.
// ===========================================================================
Poly keygen(const Ring& R, const Dist& d, Prg& prg) {
  std::vector<i64> s(R.n);
  sample_into(d, prg, s.data(), s.size());
  return R.from_centered_i64(s.data());
}

// prim/encryption/rlwe.rs encrypt: mask (uniform) drawn first, then the error.
Rlwe encrypt(const Ring& R, const Poly& sk, const Poly& encoded, const Dist& e, Prg& prg) {
  Poly mask = R.random_uniform(prg);
  std::vector<i64> es(R.n);
  sample_into(e, prg, es.data(), es.size());
  Poly err = R.from_centered_i64(es.data());
  Poly body = R.add(R.add(R.mul(mask, sk), err), encoded);
  return Rlwe{mask, body};
}

Poly decrypt_raw(const Ring& R, const Poly& sk, const Rlwe& ct) { return R.sub(ct.body, R.mul(ct.mask, sk)); }

Poly encode(const Ring& Rq, u64 p, const std::vector<u64>& pt) {
  u128 q = Rq.Q();
  u128 delta = (q + p - 1) / p;
  std::vector<u128> v(Rq.n);
  for (int i = 0; i < Rq.n; ++i) v[i] = ((u128)pt[i] * delta) % q;
  return Rq.from_u128(v);
}

std::vector<u64> decode(const Ring& Rq, u64 p, const Poly& scaled) {
  i128 q = (i128)Rq.Q(), pp = (i128)p, half = q / 2;
  std::vector<i128> c = Rq.centered(scaled);
  std::vector<u64> out(Rq.n);
  for (int i = 0; i < Rq.n; ++i) {
    i128 num = pp * c[i] + half;
    i128 r = num / q;
    if (num % q < 0) r -= 1;  // div_euclid
    i128 m = r % pp;
    if (m < 0) m += pp;
    out[i] = (u64)m;
  }
  return out;
}

Rlev encrypt_rlev(const Ring& R, const Poly& sk, const Poly& msg, u64 base, int L, const Dist& e, Prg& prg) {
  std::vector<u128> g = gadget_vector_values(R.Q(), base, L);
  Rlev out;
  for (int i = 0; i < L; ++i) {
    Poly scaled = R.mul(msg, R.scalar_const(g[i]));
    out.push_back(encrypt(R, sk, scaled, e, prg));
  }
  return out;
}

Rgsw encrypt_rgsw(const Ring& R, const Poly& sk, const Poly& msg, u64 b1, u64 b2, int L1, int L2, const Dist& e,
                  Prg& prg) {
  Poly nsm = R.neg(R.mul(sk, msg));
  Rgsw g;
  g.neg_s_m = encrypt_rlev(R, sk, nsm, b1, L1, e, prg);
  g.m = encrypt_rlev(R, sk, msg, b2, L2, e, prg);
  return g;
}

std::vector<u64> decrypt_asymmetric(const Ring& Rq3, const Poly& sk, const Poly& mask_q3, const Poly& body_q4, u64 q4,
                                    u64 p) {
  std::vector<i128> c = Rq3.centered(sk);
  std::vector<i64> c64(Rq3.n);
  for (int i = 0; i < Rq3.n; ++i) c64[i] = (i64)c[i];
  Poly skq3 = Rq3.from_centered_i64(c64.data());
  Poly prod = Rq3.mul(mask_q3, skq3);
  u128 q3 = Rq3.Q();
  Ring R4 = Ring::single(Rq3.n, q4);
  std::vector<u128> v = Rq3.to_u128(prod);
  for (auto& x : v) x = (x * q4 + q3 / 2) / q3;
  Poly sw = R4.from_u128(v);
  Poly noisy = R4.sub(body_q4, sw);
  return decode(R4, p, noisy);
}

// ===========================================================================
// Gates — prim/gates/mux.rs:75-251, rotate.rs:52-150, convert.rs:162-240.
// ===========================================================================
Rlwe cmux(const Ring& R, const RgswEval& bit, const Rlwe& c0, const Rlwe& c1, u64 b1, u64 b2) {
  Rlwe diff = rlwe_sub(R, c1, c0);
  return rlwe_add(R, c0, external_product(R, bit, diff, b1, b2));
}

void dmux(const Ring& R, const RgswEval& bit, const Rlwe& c, u64 b1, u64 b2, Rlwe& r0, Rlwe& r1) {
  Rlwe prod = external_product(R, bit, c, b1, b2);
  r0 = rlwe_sub(R, c, prod);
  r1 = prod;
}

Rlwe cmux_tree(const Ring& R, const std::vector<RgswEval>& bits, std::vector<Rlwe> in, u64 b1, u64 b2) {
  if (in.size() != ((size_t)1 << bits.size())) throw OracleError(ERR_DIM_MISMATCH, "cmux_tree: inputs != 2^m");
  size_t active = in.size();
  for (auto& bit : bits) {
    size_t half = active >> 1;
    for (size_t j = 0; j < half; ++j) in[j] = cmux(R, bit, in[2 * j], in[2 * j + 1], b1, b2);
    active = half;
  }
  return in[0];
}

std::vector<Rlwe> dmux_tree(const Ring& R, const std::vector<RgswEval>& bits, const Rlwe& input, u64 b1, u64 b2) {
  std::vector<Rlwe> out((size_t)1 << bits.size(), input);
  out[0] = input;
  for (size_t i = 0; i < bits.size(); ++i) {
    size_t active = (size_t)1 << i;
    for (size_t jj = active; jj-- > 0;) {
      Rlwe src = out[jj];
      Rlwe r0, r1;
      dmux(R, bits[i], src, b1, b2, r0, r1);
      out[2 * jj + 1] = r1;
      out[2 * jj] = r0;
    }
  }
  return out;
}

Rlwe rotate(const Ring& R, const Rlwe& c, size_t k) { return Rlwe{R.mul_x_pow(c.mask, k), R.mul_x_pow(c.body, k)}; }

Rlwe crot(const Ring& R, CRotDir dir, const std::vector<RgswEval>& bits, Rlwe ct, u64 b1, u64 b2) {
  for (size_t i = 0; i < bits.size(); ++i) {
    if (dir == CRotDir::Forward) {
      Rlwe rot = rotate(R, ct, (size_t)1 << i);
      ct = cmux(R, bits[i], ct, rot, b1, b2);
    } else {
      Rlwe nr = rlwe_neg(R, rotate(R, ct, (size_t)R.n - ((size_t)1 << i)));
      ct = cmux(R, bits[i], ct, nr, b1, b2);
    }
  }
  return ct;
}

Rgsw rlwe_to_rgsw(const Ring& R, const std::vector<Rlwe>& levels, const RlevEval& conv_key,
                  const std::vector<Rlwe>& m_rlev, u64 ck_base) {
  Rgsw g;
  for (auto& lv : levels) {
    Rlwe p = gadget_product(R, conv_key, lv.mask, ck_base);
    g.neg_s_m.push_back(Rlwe{R.add(lv.body, p.mask), p.body});
  }
  g.m = m_rlev;
  return g;
}

// ===========================================================================
// Switching — prim/switching/{mod_switch,ring_switch,rekey}.rs,
// prim/switching/kernels/mod_switch.rs:59-61.
// ===========================================================================
u128 rescale(u128 c, u128 q_src, u128 q_dst) { return (c * q_dst + q_src / 2) / q_src; }

Rlwe mod_switch_sym(const Ring& src, const Rlwe& ct, const Ring& dst) {
  u128 qs = src.Q(), qd = dst.Q();
  auto sw = [&](const Poly& a) {
    std::vector<u128> v = src.to_u128(a);
    for (auto& x : v) x = rescale(x, qs, qd);
    return dst.from_u128(v);
  };
  return Rlwe{sw(ct.mask), sw(ct.body)};
}

void mod_switch_asym(const Ring& src, const Rlwe& ct, const Ring& mask_r, const Ring& body_r, Poly& mask,
                     Poly& body) {
  u128 qs = src.Q();
  std::vector<u128> vm = src.to_u128(ct.mask), vb = src.to_u128(ct.body);
  for (auto& x : vm) x = rescale(x, qs, mask_r.Q());
  for (auto& x : vb) x = rescale(x, qs, body_r.Q());
  mask = mask_r.from_u128(vm);
  body = body_r.from_u128(vb);
}

Rgsw mod_switch_rgsw(const Ring& src, const Rgsw& g, const Ring& dst) {
  Rgsw o;
  for (auto& s : g.neg_s_m) o.neg_s_m.push_back(mod_switch_sym(src, s, dst));
  for (auto& s : g.m) o.m.push_back(mod_switch_sym(src, s, dst));
  return o;
}

Poly rekey(const Ring& src, const Poly& sk, const Ring& dst) { return dst.from_centered_i128(src.centered(sk)); }

std::vector<Rlev> gen_rsk(const Ring& R1q3, const Poly& s1, const Ring& R2q3, const Poly& s2, u64 base, int L,
                          const Dist& e, Prg& prg) {
  int D = R1q3.n / R2q3.n;
  std::vector<Rlev> out;
  for (int j = 0; j < D; ++j) {
    Poly kp;
    if (j == 0) {
      kp = project_at(R1q3, s1, R2q3.n, 0);
    } else {
      Poly rot = R1q3.mul_x_pow(s1, (size_t)R1q3.n - j);
      kp = project_at(R1q3, R1q3.neg(rot), R2q3.n, 0);
    }
    out.push_back(encrypt_rlev(R2q3, s2, kp, base, L, e, prg));
  }
  return out;
}

// prim/switching/ring_switch.rs:358-385 ring_switch_eval.
Rlwe ring_switch(const Ring& R1, const Rlwe& ct, const Ring& R2, const std::vector<RlevEval>& rsk, u64 base) {
  Poly acc_m = R2.zero();
  Poly acc_b = project_at(R1, ct.body, R2.n, 0);
  for (size_t j = 0; j < rsk.size(); ++j) {
    Poly mp = j == 0 ? project_at(R1, ct.mask, R2.n, 0) : project_at(R1, R1.mul_x_pow(ct.mask, j), R2.n, 0);
    Rlwe gp = gadget_product(R2, rsk[j], mp, base);
    R2.sub_inplace(acc_m, gp.mask);
    R2.sub_inplace(acc_b, gp.body);
  }
  return Rlwe{acc_m, acc_b};
}

// ===========================================================================
// Conversion — prim/conversion/{mlwe_ops,conv,cascade}.rs.
// ===========================================================================
// prim/conversion/mlwe_ops.rs:223-246 encrypt_lwe_raw.
Lwe encrypt_lwe_raw(const Ring& R, const Poly& sk, u128 message, const Dist& e, Prg& prg) {
  Lwe out;
  out.mask_poly = R.random_uniform(prg);
  i64 es;
  sample_into(e, prg, &es, 1);
  u128 qv = R.Q();
  u128 mv = message % qv;
  out.body.resize(R.nl);
  for (int l = 0; l < R.nl; ++l) {
    u128 acc = 0;  // prim/conversion/kernels/lwe.rs dot_residues
    u64 accr = 0;
    for (int i = 0; i < R.n; ++i) {
      acc += (u128)out.mask_poly[l * R.n + i] * sk[l * R.n + i];
      if (acc >> 120) {
        accr = R.m[l].add(accr, (u64)(acc % R.m[l].q));
        acc = 0;
      }
    }
    u64 dot = R.m[l].add(accr, (u64)(acc % R.m[l].q));
    u64 err = R.m[l].reduce_i64(es);
    u64 enc = R.m[l].reduce(mv);
    out.body[l] = R.m[l].add(R.m[l].add(dot, err), enc);
  }
  return out;
}

Lwe encrypt_lwe(const Ring& R, const Poly& sk, u64 message, u64 p, const Dist& e, Prg& prg) {
  u128 qv = R.Q();
  u128 delta = (qv + p - 1) / p;
  // encrypt_lwe draws mask, error, then encodes delta*m: same PRG order as raw.
  return encrypt_lwe_raw(R, sk, (delta * message) % qv, e, prg);
}

static Mlwe lwe_as_mlwe(const Ring& R, const Lwe& lwe) {
  Mlwe m;
  m.masks.resize(R.n);
  for (int i = 0; i < R.n; ++i) {
    Poly c(R.nl);
    for (int l = 0; l < R.nl; ++l) c[l] = lwe.mask_poly[l * R.n + i];
    m.masks[i] = c;
  }
  m.body = lwe.body;
  return m;
}

// prim/conversion/conv.rs:122-148 conv_step_eval.
Mlwe conv_step(const Ring& Rout, const Ring& Rin, const Mlwe& ct, const std::vector<RlevEval>& keys, u64 base) {
  size_t rank_in = ct.masks.size(), rank_out = rank_in / 2;
  Mlwe out;
  out.masks.assign(rank_out, Rout.zero());
  out.body = embed_at(Rin, ct.body, Rout.n, 0);
  for (int group = 0; group < 2; ++group)
    for (size_t j = 0; j < rank_out; ++j) {
      size_t idx = rank_out * group + j;
      Rlwe rl{embed_at(Rin, ct.masks[idx], Rout.n, 0), Rout.zero()};
      Rlwe sw = key_switch(Rout, keys[idx], rl, base);
      Rout.add_inplace(out.masks[j], sw.mask);
      Rout.add_inplace(out.body, sw.body);
    }
  return out;
}

// prim/conversion/conv.rs:186-236 gen_conv_step_key[_element], cascade.rs:97-120
// (steps in ascending output degree, key_idx ascending within a step).
CascadeKey gen_cascade_key(const Ring& R, const Poly& sk, u64 base, int L, const Dist& e, Prg& prg) {
  CascadeKey K;
  K.n = R.n;
  K.L = L;
  for (int nout = 2; nout <= R.n; nout <<= 1) {
    int nin = nout / 2;
    int rank_in = R.n / nin;
    int m = rank_in / 2;
    Ring Rout = R.with_n(nout);
    Ring Rin = R.with_n(nin);
    std::vector<Rlev> step;
    for (int key_idx = 0; key_idx < rank_in; ++key_idx) {
      int group = key_idx / m, j = key_idx % m;
      Poly src = embed_at(Rin, project_at(R, sk, nin, m * group + j), nout, 0);
      Poly tgt = project_at(R, sk, nout, j);
      step.push_back(encrypt_rlev(Rout, tgt, src, base, L, e, prg));
    }
    K.steps.push_back(std::move(step));
  }
  return K;
}

CascadeKeyEval cascade_key_to_eval(const Ring& R, const CascadeKey& k) {
  CascadeKeyEval E;
  E.n = k.n;
  E.L = k.L;
  int nout = 2;
  for (auto& step : k.steps) {
    Ring Rout = R.with_n(nout);
    std::vector<RlevEval> es;
    for (auto& rl : step) es.push_back(rlev_to_eval(Rout, rl));
    E.steps.push_back(std::move(es));
    nout <<= 1;
  }
  return E;
}

// prim/conversion/cascade.rs:388-404 (the macro's @chain_eval), any degree.
Rlwe lwe_to_rlwe(const Ring& R, const Lwe& lwe, const CascadeKeyEval& key, u64 base) {
  Mlwe cur = lwe_as_mlwe(R, lwe);
  int nin = 1;
  for (auto& step : key.steps) {
    Ring Rin = R.with_n(nin), Rout = R.with_n(2 * nin);
    cur = conv_step(Rout, Rin, cur, step, base);
    nin *= 2;
  }
  return Rlwe{cur.masks[0], cur.body};
}

// ===========================================================================
// Params.
// ===========================================================================
u128 Params::delta() const {
  u128 q1 = q1_1 ? (u128)q1_0 * q1_1 : (u128)q1_0;
  return (q1 + p - 1) / p;
}
static int ilog2_exact(u64 v) { return v <= 1 ? 0 : 63 - __builtin_clzll(v); }
static int ceil_log2(u64 v) { return v <= 1 ? 0 : 64 - __builtin_clzll(v - 1); }
int Params::num_dmux() const { return ilog2_exact(num_rows); }
int Params::num_cmux() const { return ilog2_exact(num_cols); }
int Params::num_crot() const { return n1 / n_rec > 1 ? ilog2_exact((u64)(n1 / n_rec)) : 0; }

// ===========================================================================
// Client — via-client/src/{client,query,decompose}.rs.
// ===========================================================================
Client client_setup(const Params& prm, const Dist& key1, const Dist& key2, const Dist& err, Prg& prg,
                    PublicKeys& pk) {
  if ((prm.num_rows & (prm.num_rows - 1)) || (prm.num_cols & (prm.num_cols - 1)) || !prm.num_rows || !prm.num_cols)
    throw OracleError(ERR_DIM_MISMATCH, "num_rows and num_cols must be powers of two");
  Client c;
  c.prm = prm;
  c.err = err;
  Ring R1 = prm.r1(), R3 = prm.r3();
  c.sk1 = keygen(R1, key1, prg);
  c.sk2 = keygen(R3, key2, prg);
  pk.cascade = gen_cascade_key(R1, c.sk1, prm.ck_base, prm.l_ck, err, prg);
  pk.conv_key = encrypt_rlev(R1, c.sk1, R1.mul(c.sk1, c.sk1), prm.ck_base, prm.l_ck, err, prg);
  Ring R3n1 = prm.r3n1();
  Poly s1q3 = rekey(R1, c.sk1, R3n1);
  pk.rsk = gen_rsk(R3n1, s1q3, R3, c.sk2, prm.b_rsk, prm.l_rsk, err, prg);
  return c;
}

std::vector<Lwe> client_query(const Client& c, u64 index, int d, Prg& prg) {
  const Params& prm = c.prm;
  u64 I = prm.num_rows, J = prm.num_cols;
  u64 nrec = (u64)d * I * J;
  if (index >= nrec) throw OracleError(ERR_INDEX_OUT_OF_RANGE, "index out of range");
  u64 group = I * J;
  u64 gamma = index / group, alpha = (index % group) / J, beta = index % J;
  Ring R1 = prm.r1();
  u128 q1 = R1.Q();
  std::vector<u128> gd = gadget_vector_values(q1, prm.b_dmux, prm.l_query);
  std::vector<u128> gc = gadget_vector_values(q1, prm.b_cmux, prm.l_query);
  int nd = ceil_log2(I), nc = ceil_log2(J), nr = ceil_log2((u64)d);
  std::vector<Lwe> out;
  auto push = [&](const std::vector<int>& bits, const std::vector<u128>& g) {
    for (int b : bits)
      for (u128 gi : g) out.push_back(encrypt_lwe_raw(R1, c.sk1, b ? gi % q1 : 0, c.err, prg));
  };
  std::vector<int> db, cb, rb;
  for (int i = 0; i < nd; ++i) db.push_back((int)((alpha >> (nd - 1 - i)) & 1));
  for (int i = 0; i < nc; ++i) cb.push_back((int)((beta >> i) & 1));
  for (int i = 0; i < nr; ++i) rb.push_back((int)((gamma >> i) & 1));
  push(db, gd);
  push(cb, gc);
  push(rb, gc);
  return out;
}

std::vector<u64> client_recover(const Client& c, const Poly& mask_q3, const Poly& body_q4) {
  return decrypt_asymmetric(c.prm.r3(), c.sk2, mask_q3, body_q4, c.prm.q4, c.prm.p);
}

// ===========================================================================
// Server — crates/via-server/src.
// ===========================================================================
PreparedKeys prepare_keys(const Params& prm, const PublicKeys& pk) {
  Ring R1 = prm.r1(), R3 = prm.r3();
  PreparedKeys k;
  k.cascade = cascade_key_to_eval(R1, pk.cascade);
  k.conv_key = rlev_to_eval(R1, pk.conv_key);
  for (auto& r : pk.rsk) k.rsk.push_back(rlev_to_eval(R3, r));
  return k;
}

template <class F>
static void parallel_for(size_t n, int threads, F f) {
  if (threads <= 1 || n < 2) {
    for (size_t i = 0; i < n; ++i) f(i);
    return;
  }
  size_t w = std::min((size_t)threads, n);
  size_t chunk = (n + w - 1) / w;
  std::vector<std::thread> ts;
  for (size_t t = 0; t < w; ++t) {
    size_t lo = t * chunk, hi = std::min(n, lo + chunk);
    if (lo >= hi) break;
    ts.emplace_back([=, &f] {
      for (size_t i = lo; i < hi; ++i) f(i);
    });
  }
  for (auto& t : ts) t.join();
}

// Record r's coefficient c: records[r * n_rec + c] (u64 layout) or the nibble
// r * n_rec + c of `packed`, low nibble first (the 4-bit packed layout).
template <class Coef>
static PreparedDb setup_db_impl(const Params& prm, Coef coef, size_t n_records, int threads) {
  u64 I = prm.num_rows, J = prm.num_cols;
  int d = prm.n1 / prm.n_rec;
  if (n_records > I * J * (u64)d)
    throw OracleError(ERR_DIM_MISMATCH, "setup: more records than DB capacity (would silently drop)");
  Ring R2 = prm.r2();
  PreparedDb db;
  db.rows = I;
  db.cols = J;
  db.cells.resize(I * J);
  parallel_for(I * J, threads, [&](size_t cell) {
    u64 i = cell / J, j = cell % J;
    std::vector<u128> v(prm.n1, 0);
    for (int k = 0; k < d; ++k) {
      u64 flat = (u64)k * I * J + i * J + j;
      if (flat >= n_records) continue;
      for (int c = 0; c < prm.n_rec; ++c)
        v[(size_t)d * c + k] = (v[(size_t)d * c + k] + coef(flat * prm.n_rec + c)) % prm.p;
    }
    db.cells[cell] = R2.to_eval(R2.from_u128(v));
  });
  return db;
}

PreparedDb setup_db(const Params& prm, const u64* records, size_t n_records, int threads) {
  return setup_db_impl(prm, [records](u64 x) { return records[x]; }, n_records, threads);
}

PreparedDb setup_db_packed(const Params& prm, const uint8_t* packed, size_t n_records, int threads) {
  return setup_db_impl(
      prm, [packed](u64 x) { return (u64)((packed[x >> 1] >> (4 * (x & 1))) & 15); }, n_records, threads);
}

std::vector<Rlwe> first_dim(const Params& prm, const std::vector<Rlwe>& switched, const PreparedDb& db, int threads) {
  if (switched.size() != db.rows) throw OracleError(ERR_DIM_MISMATCH, "first_dim: I mismatch");
  Ring R2 = prm.r2();
  std::vector<std::pair<Poly, Poly>> sel;
  for (auto& c : switched) sel.push_back({R2.to_eval(c.mask), R2.to_eval(c.body)});
  std::vector<Rlwe> out(db.cols);
  parallel_for(db.cols, threads, [&](size_t j) {
    Poly am = R2.mul_eval(db.cells[j], sel[0].first);
    Poly ab = R2.mul_eval(db.cells[j], sel[0].second);
    for (size_t i = 1; i < db.rows; ++i) {
      R2.mac_eval(am, db.cells[i * db.cols + j], sel[i].first);
      R2.mac_eval(ab, db.cells[i * db.cols + j], sel[i].second);
    }
    out[j] = Rlwe{R2.from_eval(am), R2.from_eval(ab)};
  });
  return out;
}

DecompQuery query_decomp(const Params& prm, const std::vector<Lwe>& q, const PreparedKeys& k) {
  Ring R1 = prm.r1();
  int nd = prm.num_dmux(), nc = prm.num_cmux(), nr = prm.num_crot();
  int L = prm.l_query;
  DecompQuery out;
  for (int bit = 0; bit < nd + nc + nr; ++bit) {
    std::vector<Rlwe> levels;
    for (int i = 0; i < L; ++i) levels.push_back(lwe_to_rlwe(R1, q[(size_t)bit * L + i], k.cascade, prm.ck_base));
    Rgsw g = rlwe_to_rgsw(R1, levels, k.conv_key, levels, prm.ck_base);
    if (bit < nd)
      out.dmux.push_back(g);
    else if (bit < nd + nc)
      out.cmux.push_back(g);
    else
      out.crot.push_back(g);
  }
  return out;
}

static thread_local StageTimes g_times;
const StageTimes& last_stage_times() { return g_times; }
static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

Rlwe answer_through_crot(const Params& prm, const std::vector<Lwe>& q, const PreparedKeys& k, const PreparedDb& db,
                         int threads) {
  u64 I = prm.num_rows, J = prm.num_cols;
  if ((I & (I - 1)) || (J & (J - 1)) || !I || !J)
    throw OracleError(ERR_DIM_MISMATCH, "num_rows and num_cols must be powers of two");
  if (db.rows != I) throw OracleError(ERR_DIM_MISMATCH, "prepared_db row count must equal num_rows");
  if (q.size() != prm.n_lwe()) throw OracleError(ERR_QUERY_LENGTH_MISMATCH, "query length mismatch");
  Ring R1 = prm.r1(), R2 = prm.r2();
  double t0 = now_s();
  DecompQuery dq = query_decomp(prm, q, k);
  double t1 = now_s();
  // Step 2: DMux of the trivial RLWE(0, delta) at q1 (srv/answer.rs:181-191).
  std::vector<RgswEval> dbits;
  for (auto& g : dq.dmux) dbits.push_back(rgsw_to_eval(R1, g));
  Rlwe triv{R1.zero(), R1.scalar_const(prm.delta())};
  std::vector<Rlwe> dm = dmux_tree(R1, dbits, triv, prm.b_dmux, prm.b_dmux);
  double t2 = now_s();
  std::vector<Rlwe> sw;
  for (auto& c : dm) sw.push_back(mod_switch_sym(R1, c, R2));
  double t3 = now_s();
  std::vector<Rlwe> fd = first_dim(prm, sw, db, threads);
  double t4 = now_s();
  std::vector<RgswEval> cbits, rbits;
  for (auto& g : dq.cmux) cbits.push_back(rgsw_to_eval(R2, mod_switch_rgsw(R1, g, R2)));
  Rlwe sel = cmux_tree(R2, cbits, fd, prm.b_cmux, prm.b_cmux);
  double t5 = now_s();
  for (auto& g : dq.crot) rbits.push_back(rgsw_to_eval(R2, mod_switch_rgsw(R1, g, R2)));
  Rlwe rot = crot(R2, CRotDir::SlotExtract, rbits, sel, prm.b_cmux, prm.b_cmux);
  double t6 = now_s();
  g_times.t[0] = t1 - t0;
  g_times.t[1] = t2 - t1;
  g_times.t[2] = t3 - t2;
  g_times.t[3] = t4 - t3;
  g_times.t[4] = t5 - t4;
  g_times.t[5] = t6 - t5;
  return rot;
}

void resp_comp(const Params& prm, const Rlwe& ct_q2, const std::vector<RlevEval>& rsk, Poly& mask_q3, Poly& body_q4) {
  Ring R2 = prm.r2(), R3n1 = prm.r3n1(), R3 = prm.r3(), R4 = prm.r4();
  Rlwe c3 = mod_switch_sym(R2, ct_q2, R3n1);
  Rlwe rs = ring_switch(R3n1, c3, R3, rsk, prm.b_rsk);
  mod_switch_asym(R3, rs, R3, R4, mask_q3, body_q4);
}

void answer(const Params& prm, const std::vector<Lwe>& q, const PreparedKeys& k, const PreparedDb& db, int threads,
            Poly& mask_q3, Poly& body_q4) {
  Rlwe rot = answer_through_crot(prm, q, k, db, threads);
  double t0 = now_s();
  resp_comp(prm, rot, k.rsk, mask_q3, body_q4);
  g_times.t[6] = now_s() - t0;
}

}  // namespace vo
