// C ABI of the CPU oracle — TEST INFRASTRUCTURE ONLY (tests/, smoke(), the
// bench's CPU-baseline leg). Buffers use the wire layouts of include/via_gpu.h.
#include <cstring>
#include <map>
#include <memory>
#include <thread>

#include "../include/via_gpu.h"
#include "via_oracle.hpp"

namespace vo {
std::map<std::string, std::vector<u64>> run_kat(const std::string& layer, const std::string& scenario);
}

using namespace vo;

static thread_local std::string g_err;

static Params to_params(const via_params* p) {
  Params r;
  r.n1 = (int)p->n1;
  r.n2 = (int)p->n2;
  r.n_rec = (int)p->n_rec;
  r.num_rows = p->num_rows;
  r.num_cols = p->num_cols;
  r.q1_0 = p->q1_0;
  r.q1_1 = p->q1_1;
  r.q2 = p->q2;
  r.q3 = p->q3;
  r.q4 = p->q4;
  r.p = p->p;
  r.b_dmux = p->b_dmux;
  r.b_cmux = p->b_cmux;
  r.ck_base = p->ck_base;
  r.b_rsk = p->b_rsk;
  r.l_query = (int)p->l_query;
  r.l_ck = (int)p->l_ck;
  r.l_rsk = (int)p->l_rsk;
  return r;
}

template <class F>
static int guarded(F f) {
  try {
    f();
    return 0;
  } catch (const OracleError& e) {
    g_err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_err = e.what();
    return ERR_INVALID;
  }
}

// ---- flat (de)serialisation in the include/via_gpu.h layouts -------------
static void put_poly(u64*& dst, const Poly& a) {
  std::memcpy(dst, a.data(), a.size() * 8);
  dst += a.size();
}
static Poly get_poly(const u64*& src, size_t n) {
  Poly a(src, src + n);
  src += n;
  return a;
}
static void put_rlev(u64*& dst, const Rlev& r) {
  for (auto& s : r) {
    put_poly(dst, s.mask);
    put_poly(dst, s.body);
  }
}
static Rlev get_rlev(const u64*& src, const Ring& R, int L) {
  Rlev r;
  for (int l = 0; l < L; ++l) {
    Rlwe s;
    s.mask = get_poly(src, R.size());
    s.body = get_poly(src, R.size());
    r.push_back(s);
  }
  return r;
}
static CascadeKey get_cascade(const u64*& src, const Ring& R, int L) {
  CascadeKey K;
  K.n = R.n;
  K.L = L;
  for (int nout = 2; nout <= R.n; nout <<= 1) {
    int rank_in = R.n / (nout / 2);
    Ring Ro = R.with_n(nout);
    std::vector<Rlev> step;
    for (int i = 0; i < rank_in; ++i) step.push_back(get_rlev(src, Ro, L));
    K.steps.push_back(step);
  }
  return K;
}
static std::vector<Lwe> get_query(const u64* src, const Ring& R, size_t n_lwe) {
  std::vector<Lwe> q;
  for (size_t i = 0; i < n_lwe; ++i) {
    Lwe l;
    l.mask_poly = get_poly(src, R.size());
    l.body = get_poly(src, R.nl);
    q.push_back(l);
  }
  return q;
}

struct OracleServer {
  Params prm;
  PreparedKeys keys;
  PreparedDb db;
  CascadeKey cascade;                              // coefficient form, for the VIA-B repack keys
  std::vector<std::vector<RlevEval>> repack_keys;  // derived on the first answer_batch
};

extern "C" {

const char* vo_last_error(void) { return g_err.c_str(); }

void vo_shake256(const uint8_t* in, size_t inlen, uint8_t* out, size_t outlen) { shake256(in, inlen, out, outlen); }

// Runs one replayed reference KAT and copies the named output. Returns the
// number of values (or -code on error; -1 if the name is unknown).
long vo_kat(const char* layer, const char* scenario, const char* name, uint64_t* out, size_t cap) {
  long n = -1;
  int rc = guarded([&] {
    auto o = run_kat(layer, scenario);
    auto it = o.find(name);
    if (it == o.end()) return;
    n = (long)it->second.size();
    std::memcpy(out, it->second.data(), std::min((size_t)n, cap) * 8);
  });
  return rc ? -rc : n;
}

// Client::setup (cli/client.rs:89-180) with ternary keys and errors; writes the
// public keys in wire layout. Returns an opaque client or NULL.
void* vo_client_setup(const via_params* p, const uint8_t* seed, size_t seedlen, uint64_t* cascade, uint64_t* conv,
                      uint64_t* rsk) {
  Client* out = nullptr;
  guarded([&] {
    Params prm = to_params(p);
    Prg prg(seed, seedlen);
    PublicKeys pk;
    Dist T = Dist::ternary();
    auto c = std::make_unique<Client>(client_setup(prm, T, T, T, prg, pk));
    u64* d = cascade;
    for (auto& st : pk.cascade.steps)
      for (auto& rl : st) put_rlev(d, rl);
    d = conv;
    put_rlev(d, pk.conv_key);
    d = rsk;
    for (auto& r : pk.rsk) put_rlev(d, r);
    out = c.release();
  });
  return out;
}

// Client::query / batch_query (cli/client.rs:183-220): `d` is n1 / n_rec.
int vo_client_query(void* c, uint64_t index, uint32_t d, const uint8_t* seed, size_t seedlen, uint64_t* out) {
  return guarded([&] {
    Client* cl = (Client*)c;
    Prg prg(seed, seedlen);
    std::vector<Lwe> q = client_query(*cl, index, (int)d, prg);
    u64* dst = out;
    for (auto& l : q) {
      put_poly(dst, l.mask_poly);
      put_poly(dst, l.body);
    }
  });
}

// Client::recover (cli/client.rs:222-237): n2 plaintext coefficients.
int vo_client_recover(void* c, const uint64_t* mask, const uint64_t* body, uint64_t* out) {
  return guarded([&] {
    Client* cl = (Client*)c;
    int n2 = cl->prm.n2;
    Poly m(mask, mask + n2), b(body, body + n2);
    std::vector<u64> r = client_recover(*cl, m, b);
    std::memcpy(out, r.data(), r.size() * 8);
  });
}

// The client's secret keys (S1 at q1, nl * n1 residues; S2 at q3, n2 residues),
// for the device client's parity tests.
void vo_client_secret(void* c, uint64_t* sk1, uint64_t* sk2) {
  const Client* cl = (const Client*)c;
  std::memcpy(sk1, cl->sk1.data(), cl->sk1.size() * 8);
  std::memcpy(sk2, cl->sk2.data(), cl->sk2.size() * 8);
}

void vo_client_free(void* c) { delete (Client*)c; }

// Server::setup (srv/answer.rs:486-528). Records: n_rec u64 coefficients each.
// records: u64 coefficients (packed == 0) or 4-bit coefficients two per byte,
// low nibble first (packed == 1).
static void* server_setup(const via_params* p, const uint64_t* cascade, const uint64_t* conv, const uint64_t* rsk,
                          const void* records, int packed, size_t n_records, int threads) {
  OracleServer* out = nullptr;
  guarded([&] {
    auto s = std::make_unique<OracleServer>();
    s->prm = to_params(p);
    const Params& prm = s->prm;
    Ring R1 = prm.r1(), R3 = prm.r3();
    PublicKeys pk;
    const u64* src = cascade;
    pk.cascade = get_cascade(src, R1, prm.l_ck);
    src = conv;
    pk.conv_key = get_rlev(src, R1, prm.l_ck);
    src = rsk;
    for (int j = 0; j < prm.d(); ++j) pk.rsk.push_back(get_rlev(src, R3, prm.l_rsk));
    s->keys = prepare_keys(prm, pk);
    s->cascade = pk.cascade;
    s->db = packed ? setup_db_packed(prm, (const uint8_t*)records, n_records, threads)
                   : setup_db(prm, (const u64*)records, n_records, threads);
    out = s.release();
  });
  return out;
}

void* vo_server_setup(const via_params* p, const uint64_t* cascade, const uint64_t* conv, const uint64_t* rsk,
                      const uint64_t* records, size_t n_records, int threads) {
  return server_setup(p, cascade, conv, rsk, records, 0, n_records, threads);
}

void* vo_server_setup_packed(const via_params* p, const uint64_t* cascade, const uint64_t* conv, const uint64_t* rsk,
                             const uint8_t* packed, size_t n_records, int threads) {
  return server_setup(p, cascade, conv, rsk, packed, 1, n_records, threads);
}

int vo_server_answer(void* sv, const uint64_t* query, size_t n_lwe, uint64_t* mask, uint64_t* body, int threads) {
  return guarded([&] {
    OracleServer* s = (OracleServer*)sv;
    Ring R1 = s->prm.r1();
    std::vector<Lwe> q = get_query(query, R1, n_lwe);
    Poly m, b;
    answer(s->prm, q, s->keys, s->db, threads, m, b);
    std::memcpy(mask, m.data(), m.size() * 8);
    std::memcpy(body, b.data(), b.size() * 8);
  });
}

// Server::answer_batch (srv/batch.rs:72-163): n_queries = T = n2 / n_rec queries
// of n_lwe LWEs each, back to back; one answer.
int vo_server_answer_batch(void* sv, const uint64_t* queries, size_t n_queries, size_t n_lwe, uint64_t* mask,
                           uint64_t* body, int threads) {
  return guarded([&] {
    OracleServer* s = (OracleServer*)sv;
    Ring R1 = s->prm.r1();
    const size_t per = n_lwe * (size_t)R1.nl * (s->prm.n1 + 1);
    std::vector<std::vector<Lwe>> qs;
    for (size_t b = 0; b < n_queries; ++b) qs.push_back(get_query(queries + b * per, R1, n_lwe));
    if (s->repack_keys.empty()) s->repack_keys = repack_keys(s->prm, s->cascade);
    Poly m, bd;
    answer_batch(s->prm, qs, s->keys, s->repack_keys, s->db, threads, m, bd);
    std::memcpy(mask, m.data(), m.size() * 8);
    std::memcpy(body, bd.data(), bd.size() * 8);
  });
}

// Steps 1..6 only (srv/answer.rs:83-228): the CRot output RLWE at (q2, n1).
int vo_server_answer_through_crot(void* sv, const uint64_t* query, size_t n_lwe, uint64_t* out, int threads) {
  return guarded([&] {
    OracleServer* s = (OracleServer*)sv;
    std::vector<Lwe> q = get_query(query, s->prm.r1(), n_lwe);
    Rlwe r = answer_through_crot(s->prm, q, s->keys, s->db, threads);
    u64* d = out;
    put_poly(d, r.mask);
    put_poly(d, r.body);
  });
}

// FirstDim (srv/first_dim.rs:94-184): I RLWEs at (q2, n1) -> J RLWEs.
int vo_server_first_dim(void* sv, const uint64_t* switched, uint64_t* out, int threads) {
  return guarded([&] {
    OracleServer* s = (OracleServer*)sv;
    int n = s->prm.n1;
    std::vector<Rlwe> in;
    const u64* src = switched;
    for (u64 i = 0; i < s->prm.num_rows; ++i) {
      Rlwe c;
      c.mask = get_poly(src, n);
      c.body = get_poly(src, n);
      in.push_back(c);
    }
    std::vector<Rlwe> r = first_dim(s->prm, in, s->db, threads);
    u64* d = out;
    for (auto& c : r) {
      put_poly(d, c.mask);
      put_poly(d, c.body);
    }
  });
}

}  // extern "C"

// ---- primitives (include/via_gpu.h via_ntt_*_dev, via_external_product_dev,
// via_key_switch_dev): the reference operations on flat buffers.
static Ring prim_ring(uint64_t q0, uint64_t q1, int n) { return q1 ? Ring::rns(n, q0, q1) : Ring::single(n, q0); }

template <class F>
static void prim_parallel(size_t count, int threads, F f) {
  threads = std::max(1, std::min<int>(threads, (int)count));
  std::vector<std::thread> ts;
  for (int t = 0; t < threads; ++t)
    ts.emplace_back([&, t] {
      for (size_t c = t; c < count; c += threads) f(c);
    });
  for (auto& th : ts) th.join();
}

extern "C" {

// gadget_scale_into + gadget_extract_lsb_into (encryption/gadget.rs:115-190) per
// coefficient (nl residues each): count * L digits, LSB first.
int vo_gadget_digits(uint64_t q0, uint64_t q1, uint64_t base, int L, const uint64_t* coeffs, size_t count,
                     int64_t* out) {
  return guarded([&] {
    Ring R = q1 ? Ring::rns(1, q0, q1) : Ring::single(1, q0);
    std::vector<i128> scratch;
    std::vector<i64> dig;
    for (size_t i = 0; i < count; ++i) {
      Poly x(coeffs + i * R.nl, coeffs + (i + 1) * R.nl);
      gadget_scale_into(R, x, base, L, scratch);
      for (int k = 0; k < L; ++k) {
        gadget_extract_lsb_into(base, scratch, dig);
        out[i * L + k] = dig[0];
      }
    }
  });
}

// algebra/ring/ntt.rs:305-399 on [count][nl][n], in place.
int vo_ntt(uint64_t q0, uint64_t q1, int n, int inverse, uint64_t* data, size_t count) {
  return guarded([&] {
    Ring R = prim_ring(q0, q1, n);
    if (!R.eval_is_ntt()) throw OracleError(ERR_INVALID, "ring is not NTT-friendly");
    for (size_t c = 0; c < count; ++c) {
      u64* p = data + c * R.size();
      Poly a(p, p + R.size());
      Poly r = inverse ? R.from_eval(a) : R.to_eval(a);
      std::memcpy(p, r.data(), r.size() * 8);
    }
  });
}

// encryption/rgsw.rs:108-121 for `count` pairs, one gadget for both halves.
int vo_external_product(uint64_t q0, uint64_t q1, int n, uint64_t base, int L, const uint64_t* rgsw,
                        const uint64_t* rlwe, size_t count, uint64_t* out, int threads) {
  return guarded([&] {
    Ring R = prim_ring(q0, q1, n);
    const size_t per = R.size();
    prim_parallel(count, threads, [&](size_t c) {
      const u64* src = rgsw + c * 2 * L * 2 * per;
      Rgsw g;
      g.neg_s_m = get_rlev(src, R, L);
      g.m = get_rlev(src, R, L);
      const u64* cs = rlwe + c * 2 * per;
      Rlwe ct{get_poly(cs, per), get_poly(cs, per)};
      Rlwe r = external_product(R, rgsw_to_eval(R, g), ct, base, base);
      u64* d = out + c * 2 * per;
      put_poly(d, r.mask);
      put_poly(d, r.body);
    });
  });
}

// key_switch (encryption/keyswitch.rs:99-102) of X^k * ct (element.rs:328).
int vo_key_switch(uint64_t q0, uint64_t q1, int n, uint64_t base, int L, const uint64_t* key, const uint64_t* rlwe,
                  const uint64_t* shifts, size_t count, uint64_t* out, int threads) {
  return guarded([&] {
    Ring R = prim_ring(q0, q1, n);
    const size_t per = R.size();
    const u64* ks = key;
    const RlevEval K = rlev_to_eval(R, get_rlev(ks, R, L));
    prim_parallel(count, threads, [&](size_t c) {
      const u64* cs = rlwe + c * 2 * per;
      Rlwe ct{get_poly(cs, per), get_poly(cs, per)};
      Rlwe rot{R.mul_x_pow(ct.mask, shifts[c]), R.mul_x_pow(ct.body, shifts[c])};
      Rlwe r = key_switch(R, K, rot, base);
      u64* d = out + c * 2 * per;
      put_poly(d, r.mask);
      put_poly(d, r.body);
    });
  });
}

// Stage-by-stage intermediates in the include/via_gpu.h via_debug_stage layout.
int vo_server_debug_stage(void* sv, const uint64_t* query, size_t n_lwe, int stage, uint64_t* out, int threads) {
  return guarded([&] {
    OracleServer* s = (OracleServer*)sv;
    const Params& prm = s->prm;
    Ring R1 = prm.r1(), R2 = prm.r2();
    std::vector<Lwe> q = get_query(query, R1, n_lwe);
    u64* d = out;
    auto put_rlwe = [&](const Rlwe& c) {
      put_poly(d, c.mask);
      put_poly(d, c.body);
    };
    if (stage == 1) {
      for (auto& l : q) put_rlwe(lwe_to_rlwe(R1, l, s->keys.cascade, prm.ck_base));
      return;
    }
    DecompQuery dq = query_decomp(prm, q, s->keys);
    if (stage == 2) {
      for (auto* grp : {&dq.dmux, &dq.cmux, &dq.crot})
        for (auto& g : *grp) {
          put_rlev(d, g.neg_s_m);
          put_rlev(d, g.m);
        }
      return;
    }
    std::vector<RgswEval> dbits;
    for (auto& g : dq.dmux) dbits.push_back(rgsw_to_eval(R1, g));
    Rlwe triv{R1.zero(), R1.scalar_const(prm.delta())};
    std::vector<Rlwe> dm = dmux_tree(R1, dbits, triv, prm.b_dmux, prm.b_dmux);
    if (stage == 3) {
      for (auto& c : dm) put_rlwe(c);
      return;
    }
    std::vector<Rlwe> sw;
    for (auto& c : dm) sw.push_back(mod_switch_sym(R1, c, R2));
    if (stage == 4) {
      for (auto& c : sw) put_rlwe(c);
      return;
    }
    std::vector<Rlwe> fd = first_dim(prm, sw, s->db, threads);
    if (stage == 5) {
      for (auto& c : fd) put_rlwe(c);
      return;
    }
    std::vector<RgswEval> cbits, rbits;
    for (auto& g : dq.cmux) cbits.push_back(rgsw_to_eval(R2, mod_switch_rgsw(R1, g, R2)));
    Rlwe sel = cmux_tree(R2, cbits, fd, prm.b_cmux, prm.b_cmux);
    if (stage == 6) {
      put_rlwe(sel);
      return;
    }
    for (auto& g : dq.crot) rbits.push_back(rgsw_to_eval(R2, mod_switch_rgsw(R1, g, R2)));
    put_rlwe(crot(R2, CRotDir::SlotExtract, rbits, sel, prm.b_cmux, prm.b_cmux));
  });
}

// Seconds spent in steps 1..7 by the last vo_server_answer on this thread.
void vo_stage_times(double* out7) {
  const StageTimes& t = last_stage_times();
  for (int i = 0; i < 7; ++i) out7[i] = t.t[i];
}

void vo_server_free(void* s) { delete (OracleServer*)s; }

}  // extern "C"
