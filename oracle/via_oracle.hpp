// CPU oracle for the VIA server answer path — TEST INFRASTRUCTURE ONLY.
//
// A plain C++17 restatement of the reference (roynalnaruto/via-rs, pure Rust)
// arithmetic on the server answer path and of the client-side code that makes
// its seeded inputs. It is the checker for the CUDA path and the timed CPU
// baseline; nothing in the product links it. Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg may load it.
//
// Parity is pinned against the reference's own known-answer constants
// (crates/via-primitives/tests/data/layer{3,4,5}_kats.rs,
// crates/via-integration/tests/data/layer6_kats.rs), its PRG/sampler unit
// vectors, and its end-to-end "recover == record" property.
//
// Every function cites the reference file:line it follows (paths relative to the
// reference repository root; `prim/` = crates/via-primitives/src/).
#pragma once
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace vo {

using u8 = uint8_t;
using u32 = uint32_t;
using u64 = uint64_t;
using i64 = int64_t;
using u128 = unsigned __int128;
using i128 = __int128;

struct OracleError : std::runtime_error {
  int code;
  OracleError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
// Error codes: via_protocol::ViaError discriminant + 1 (proto/error.rs:20-64),
// the same numbering as include/via_gpu.h.
enum : int {
  ERR_INDEX_OUT_OF_RANGE = 2,
  ERR_QUERY_LENGTH_MISMATCH = 3,
  ERR_DIM_MISMATCH = 7,
  ERR_INVALID = 100,
};

// ---------------------------------------------------------------------------
// SHAKE-256 counter-mode PRG — prim/sampling/prg.rs:57-205.
// block_i = SHAKE256(seed || le64(i))[0..136]; bytes are served in order.
// ---------------------------------------------------------------------------
void shake256(const u8* in, size_t inlen, u8* out, size_t outlen);

struct Prg {
  u8 seed[64];
  size_t seed_len = 0;
  u64 counter = 0;
  u8 buf[136];
  size_t pos = 136;
  Prg(const void* s, size_t len);
  explicit Prg(const std::string& s) : Prg(s.data(), s.size()) {}
  void refill();
  void fill(u8* out, size_t n);
  // prim/sampling/prg.rs uniform_below: rejection on the low bitlen(bound) bits.
  u64 uniform_below(u64 bound);
};

// prim/sampling/distribution.rs:88-118 (Ternary / BoundedUniform). The Gaussian
// arm is not reproduced: no server-path test uses it and no KAT pins it.
struct Dist {
  int kind = 0;  // 0 = ternary, 1 = bounded uniform in [-bound, bound]
  u32 bound = 0;
  static Dist ternary() { return Dist{0, 0}; }
};
void sample_into(const Dist& d, Prg& prg, i64* out, size_t n);

// ---------------------------------------------------------------------------
// Modulus — prim/algebra/zq/modulus.rs (ConstModulus / PowerOfTwoModulus /
// DynModulus) with Barrett mu = floor(2^128/q) (+1 if q | 2^128),
// prim/algebra/zq/reduce.rs:59-147.
// ---------------------------------------------------------------------------
struct Mod {
  u64 q = 0;
  u128 mu = 0;
  int log2q = -1;  // >= 0 when q is a power of two (mask reduction)
  Mod() = default;
  explicit Mod(u64 q_);
  u64 reduce(u128 x) const;
  u64 add(u64 a, u64 b) const { u64 s = a + b; return s >= q ? s - q : s; }
  u64 sub(u64 a, u64 b) const { return a >= b ? a - b : a + (q - b); }
  u64 neg(u64 a) const { return a == 0 ? 0 : q - a; }
  u64 mul(u64 a, u64 b) const { return reduce((u128)a * b); }
  u64 reduce_i64(i64 x) const;
};

// ---------------------------------------------------------------------------
// Ring: R_{n,Q} with Q a single modulus (reference `Poly`) or a two-prime RNS
// basis (reference `PolyRns`, prim/algebra/ring/rns_element.rs:44-54).
// A polynomial is a flat vector of nl*n u64 residues, limb-major (limb 0 first),
// exactly the reference's in-memory layout.
// ---------------------------------------------------------------------------
using Poly = std::vector<u64>;

struct NttTable;  // negacyclic NTT tables for (q, n)

struct Ring {
  int n = 0;
  int nl = 1;  // 1 = single modulus, 2 = two-prime RNS
  Mod m[2];
  u64 q0inv_mod_q1 = 0;          // prim/algebra/rns/basis.rs Q0_INV_MOD_Q1
  const NttTable* ntt[2] = {nullptr, nullptr};  // non-null iff NTT-friendly

  static Ring single(int n, u64 q);
  static Ring rns(int n, u64 q0, u64 q1);
  Ring with_n(int n2) const;  // same moduli, another degree
  u128 Q() const { return nl == 1 ? (u128)m[0].q : (u128)m[0].q * m[1].q; }
  size_t size() const { return (size_t)nl * n; }
  bool eval_is_ntt() const { return ntt[0] != nullptr; }

  Poly zero() const { return Poly(size(), 0); }
  Poly add(const Poly& a, const Poly& b) const;
  Poly sub(const Poly& a, const Poly& b) const;
  Poly neg(const Poly& a) const;
  void add_inplace(Poly& a, const Poly& b) const;
  void sub_inplace(Poly& a, const Poly& b) const;
  // Negacyclic product in coefficient form (schoolbook or NTT; both exact).
  Poly mul(const Poly& a, const Poly& b) const;
  // Evaluation form (prim/algebra/ring/ntt_abstraction.rs): NTT when every limb
  // is NTT-friendly at this n, else the identity (the schoolbook backend).
  Poly to_eval(const Poly& a) const;
  Poly from_eval(const Poly& a) const;
  void mac_eval(Poly& acc, const Poly& a, const Poly& b) const;  // acc += a (*) b
  Poly mul_eval(const Poly& a, const Poly& b) const;

  Poly from_u128(const std::vector<u128>& v) const;      // reduce each value
  std::vector<u128> to_u128(const Poly& a) const;         // CRT reconstruct
  std::vector<i128> centered(const Poly& a) const;        // v <= Q/2 ? v : v - Q
  Poly from_centered_i64(const i64* s) const;
  Poly from_centered_i128(const std::vector<i128>& s) const;
  Poly random_uniform(Prg& prg) const;  // per coeff: limb0 then limb1
  Poly mul_x_pow(const Poly& a, size_t k) const;
  Poly scalar_const(u128 c) const;  // the constant polynomial c (reduced)
};

Poly embed_at(const Ring& src, const Poly& a, int n_large, int slot);
Poly project_at(const Ring& src, const Poly& a, int n_small, int slot);

// ---------------------------------------------------------------------------
// Ciphertext types — prim/encryption/types.rs:148-251.
// ---------------------------------------------------------------------------
struct Rlwe {
  Poly mask, body;
};
using Rlev = std::vector<Rlwe>;  // samples[0] pairs with the largest gadget entry
struct RlevEval {
  std::vector<Poly> mask, body;  // eval-form images of each sample
};
struct Rgsw {
  Rlev neg_s_m, m;
};
struct RgswEval {
  RlevEval neg_s_m, m;
};
struct Mlwe {  // rank-r MLWE over degree-n polys (reference MLWECiphertext)
  std::vector<Poly> masks;
  Poly body;
};

Rlwe rlwe_add(const Ring& R, const Rlwe& a, const Rlwe& b);
Rlwe rlwe_sub(const Ring& R, const Rlwe& a, const Rlwe& b);
Rlwe rlwe_neg(const Ring& R, const Rlwe& a);
RlevEval rlev_to_eval(const Ring& R, const Rlev& k);
RgswEval rgsw_to_eval(const Ring& R, const Rgsw& g);

// ---------------------------------------------------------------------------
// Gadget — prim/encryption/gadget.rs; wide arithmetic prim/algebra/wide.rs.
// ---------------------------------------------------------------------------
u128 round_mul_div_u128(u128 num_abs, u128 scale, u128 divisor);
std::vector<u128> gadget_vector_values(u128 Q, u64 base, int L);
void gadget_scale_into(const Ring& R, const Poly& x, u64 base, int L, std::vector<i128>& scratch);
void gadget_extract_lsb_into(u64 base, std::vector<i128>& scratch, std::vector<i64>& out);
// RLev gadget product (prim/encryption/rlev.rs:259-283): digit k (LSB-first)
// pairs with samples[L-1-k].
Rlwe gadget_product(const Ring& R, const RlevEval& key, const Poly& x, u64 base);
Rlwe gadget_product_coeff(const Ring& R, const Rlev& key, const Poly& x, u64 base);
Rlwe key_switch(const Ring& R, const RlevEval& key, const Rlwe& ct, u64 base);
Rlwe external_product(const Ring& R, const RgswEval& g, const Rlwe& ct, u64 b1, u64 b2);

// ---------------------------------------------------------------------------
// Secret-key side — prim/encryption/{rlwe,rlev,rgsw}.rs.
// ---------------------------------------------------------------------------
Poly keygen(const Ring& R, const Dist& d, Prg& prg);
Rlwe encrypt(const Ring& R, const Poly& sk, const Poly& encoded, const Dist& e, Prg& prg);
Poly decrypt_raw(const Ring& R, const Poly& sk, const Rlwe& ct);
Poly encode(const Ring& Rq, u64 p, const std::vector<u64>& pt);
std::vector<u64> decode(const Ring& Rq, u64 p, const Poly& scaled);
Rlev encrypt_rlev(const Ring& R, const Poly& sk, const Poly& msg, u64 base, int L, const Dist& e, Prg& prg);
Rgsw encrypt_rgsw(const Ring& R, const Poly& sk, const Poly& msg, u64 b1, u64 b2, int L1, int L2,
                  const Dist& e, Prg& prg);
// prim/encryption/rlwe.rs:187-240. sk2 lives at q3 (single modulus).
std::vector<u64> decrypt_asymmetric(const Ring& Rq3, const Poly& sk, const Poly& mask_q3,
                                    const Poly& body_q4, u64 q4, u64 p);

// ---------------------------------------------------------------------------
// Gates — prim/gates/{mux,rotate,convert}.rs.
// ---------------------------------------------------------------------------
Rlwe cmux(const Ring& R, const RgswEval& bit, const Rlwe& c0, const Rlwe& c1, u64 b1, u64 b2);
void dmux(const Ring& R, const RgswEval& bit, const Rlwe& c, u64 b1, u64 b2, Rlwe& r0, Rlwe& r1);
Rlwe cmux_tree(const Ring& R, const std::vector<RgswEval>& bits, std::vector<Rlwe> inputs, u64 b1, u64 b2);
std::vector<Rlwe> dmux_tree(const Ring& R, const std::vector<RgswEval>& bits, const Rlwe& input, u64 b1,
                            u64 b2);
Rlwe rotate(const Ring& R, const Rlwe& c, size_t k);
enum class CRotDir { Forward, SlotExtract };
Rlwe crot(const Ring& R, CRotDir dir, const std::vector<RgswEval>& bits, Rlwe ct, u64 b1, u64 b2);
Rgsw rlwe_to_rgsw(const Ring& R, const std::vector<Rlwe>& levels, const RlevEval& conv_key,
                  const std::vector<Rlwe>& m_rlev, u64 ck_base);

// ---------------------------------------------------------------------------
// Switching — prim/switching/{mod_switch,ring_switch,rekey}.rs.
// ---------------------------------------------------------------------------
u128 rescale(u128 c, u128 q_src, u128 q_dst);  // (c*q_dst + q_src/2) / q_src
Rlwe mod_switch_sym(const Ring& src, const Rlwe& ct, const Ring& dst);
void mod_switch_asym(const Ring& src, const Rlwe& ct, const Ring& mask_r, const Ring& body_r, Poly& mask,
                     Poly& body);
Rgsw mod_switch_rgsw(const Ring& src, const Rgsw& g, const Ring& dst);
Poly rekey(const Ring& src, const Poly& sk, const Ring& dst);
std::vector<Rlev> gen_rsk(const Ring& R1q3, const Poly& s1, const Ring& R2q3, const Poly& s2, u64 base, int L,
                          const Dist& e, Prg& prg);
Rlwe ring_switch(const Ring& R1, const Rlwe& ct, const Ring& R2, const std::vector<RlevEval>& rsk, u64 base);

// ---------------------------------------------------------------------------
// Conversion — prim/conversion/{conv,cascade,mlwe_ops}.rs.
// ---------------------------------------------------------------------------
// An LWE ciphertext of dimension n = MLWE<n,1>: masks[i] = coefficient i of a
// uniform degree-n poly. Stored as that poly (nl*n) plus a body (nl values).
struct Lwe {
  Poly mask_poly;  // nl*n, limb-major
  Poly body;       // nl values
};
Lwe encrypt_lwe_raw(const Ring& R, const Poly& sk, u128 message, const Dist& e, Prg& prg);
Lwe encrypt_lwe(const Ring& R, const Poly& sk, u64 message, u64 p, const Dist& e, Prg& prg);
// Cascade key: steps k = 1..log2 n ascending; step k holds RANK_IN = n >> (k-1)
// RLevs at degree 2^k (reference gen_conv_step_key order).
struct CascadeKey {
  int n = 0, L = 0;
  std::vector<std::vector<Rlev>> steps;
};
struct CascadeKeyEval {
  int n = 0, L = 0;
  std::vector<std::vector<RlevEval>> steps;
};
CascadeKey gen_cascade_key(const Ring& R, const Poly& sk, u64 base, int L, const Dist& e, Prg& prg);
CascadeKeyEval cascade_key_to_eval(const Ring& R, const CascadeKey& k);
Mlwe conv_step(const Ring& Rout, const Ring& Rin, const Mlwe& ct, const std::vector<RlevEval>& keys, u64 base);
Rlwe lwe_to_rlwe(const Ring& R, const Lwe& lwe, const CascadeKeyEval& key, u64 base);

// ---------------------------------------------------------------------------
// Protocol parameters — proto/params.rs:59-125 plus the DB dims and N_REC.
// ---------------------------------------------------------------------------
struct Params {
  int n1 = 0, n2 = 0, n_rec = 0;
  u64 num_rows = 0, num_cols = 0;
  u64 q1_0 = 0, q1_1 = 0;  // q1_1 == 0: single-modulus q1
  u64 q2 = 0, q3 = 0, q4 = 0, p = 0;
  u64 b_dmux = 0, b_cmux = 0, ck_base = 0, b_rsk = 0;
  int l_query = 0, l_ck = 0, l_rsk = 0;
  int d() const { return n1 / n2; }
  Ring r1() const { return q1_1 ? Ring::rns(n1, q1_0, q1_1) : Ring::single(n1, q1_0); }
  Ring r2() const { return Ring::single(n1, q2); }
  Ring r3n1() const { return Ring::single(n1, q3); }
  Ring r3() const { return Ring::single(n2, q3); }
  Ring r4() const { return Ring::single(n2, q4); }
  u128 delta() const;  // ceil(q1 / p) (proto/params.rs:376)
  int num_dmux() const;
  int num_cmux() const;
  int num_crot() const;  // log2(n1 / n_rec)
  size_t n_lwe() const { return (size_t)(num_dmux() + num_cmux() + num_crot()) * l_query; }
};

struct PublicKeys {
  CascadeKey cascade;
  Rlev conv_key;           // RLev_{S1}(S1^2), L_CK samples at q1
  std::vector<Rlev> rsk;   // D RLevs at (q3, n2)
};

struct Client {
  Params prm;
  Poly sk1, sk2;
  Dist err;
};
// via-client/src/client.rs:89-180 (keygen order: S1, S2, cascade key, conv key, RSK).
Client client_setup(const Params& prm, const Dist& key1, const Dist& key2, const Dist& err, Prg& prg,
                    PublicKeys& pk);
// via-client/src/query.rs:75-130; d = n1 / n_rec crot range.
std::vector<Lwe> client_query(const Client& c, u64 index, int d, Prg& prg);
std::vector<u64> client_recover(const Client& c, const Poly& mask_q3, const Poly& body_q4);

// ---------------------------------------------------------------------------
// Server — crates/via-server/src/*.rs.
// ---------------------------------------------------------------------------
struct PreparedKeys {
  CascadeKeyEval cascade;
  RlevEval conv_key;
  std::vector<RlevEval> rsk;
};
PreparedKeys prepare_keys(const Params& prm, const PublicKeys& pk);

struct PreparedDb {
  u64 rows = 0, cols = 0;
  std::vector<Poly> cells;  // rows*cols eval-form polys at q2, row-major
};
// setup_db (srv/setup_db.rs:39-75) + PreparedDb::from_encoded (srv/prepared_db.rs:57-85).
// records: n_records polynomials of degree n_rec, coefficients in [0, p).
PreparedDb setup_db(const Params& prm, const u64* records, size_t n_records, int threads);
// The same from 4-bit records packed two per byte, low nibble first.
PreparedDb setup_db_packed(const Params& prm, const uint8_t* packed, size_t n_records, int threads);
// srv/first_dim.rs:94-184; threads > 1 fans the J loop like the reference.
std::vector<Rlwe> first_dim(const Params& prm, const std::vector<Rlwe>& switched, const PreparedDb& db,
                            int threads);

struct DecompQuery {
  std::vector<Rgsw> dmux, cmux, crot;
};
DecompQuery query_decomp(const Params& prm, const std::vector<Lwe>& q, const PreparedKeys& k);
// srv/answer.rs:83-228 — steps 1..6, returns the CRot output at q2.
Rlwe answer_through_crot(const Params& prm, const std::vector<Lwe>& q, const PreparedKeys& k,
                         const PreparedDb& db, int threads);
// srv/resp_comp.rs:46-76.
void resp_comp(const Params& prm, const Rlwe& ct_q2, const std::vector<RlevEval>& rsk, Poly& mask_q3,
               Poly& body_q4);
// srv/answer.rs:289-354.
void answer(const Params& prm, const std::vector<Lwe>& q, const PreparedKeys& k, const PreparedDb& db,
            int threads, Poly& mask_q3, Poly& body_q4);

// ---------------------------------------------------------------------------
// VIA-B — oracle_batch.cpp (conversion/extract.rs, conversion/repack.rs,
// srv/batch.rs). The batch size is T = n2 / n_rec (the record-fit boundary).
// ---------------------------------------------------------------------------
Mlwe extr(const Ring& R, const Rlwe& ct, int g);
Mlwe mlwes_to_mlwe(const Ring& Rout, const Ring& Rin, const Mlwe& a, const Mlwe& b, const std::vector<RlevEval>& keys,
                   u64 base);
std::vector<std::vector<RlevEval>> repack_keys(const Params& prm, const CascadeKey& ck);
Rlwe repack(const Params& prm, const std::vector<Rlwe>& rotated, const std::vector<std::vector<RlevEval>>& keys);
void answer_batch(const Params& prm, const std::vector<std::vector<Lwe>>& queries, const PreparedKeys& k,
                  const std::vector<std::vector<RlevEval>>& rkeys, const PreparedDb& db, int threads, Poly& mask_q3,
                  Poly& body_q4);

// Stage timings (seconds) of the last answer() call on this thread.
struct StageTimes {
  double t[8];
};
const StageTimes& last_stage_times();

}  // namespace vo
