// CPU oracle, part 3: replays of the reference's known-answer tests.
// Test infrastructure only (see via_oracle.hpp).
//
// Each scenario restates one reference test function with the same PRG seed
// labels, the same draw order and the same parameters, and returns its outputs
// by the names the reference's generated KAT constants use. The Python tests
// compare them with tests/golden/kats.json.
#include <cstring>
#include <map>

#include "via_oracle.hpp"

namespace vo {

using Outputs = std::map<std::string, std::vector<u64>>;

static std::vector<u64> coeffs(const Ring& R, const Poly& a) {
  std::vector<u128> v = R.to_u128(a);
  return std::vector<u64>(v.begin(), v.end());
}

// ---- crates/via-primitives/tests/layer3_kats.rs ---------------------------
static Outputs layer3(const std::string& name) {
  const int N1 = 64, N2 = 16, DEPTH = 8;
  const u64 BASE = 4;
  Ring q2 = Ring::single(N1, 1ull << 32), q3 = Ring::single(N1, 1ull << 16), q4 = Ring::single(N1, 1ull << 12);
  Ring q3s = Ring::single(N2, 1ull << 16), q4s = Ring::single(N2, 1ull << 12);
  Dist T = Dist::ternary();
  Outputs o;
  if (name == "mod_switch_sym") {  // kat_mod_switch_sym
    Prg prg("layer3-kat-mod-switch-sym");
    Rlwe ct;
    ct.mask = q2.random_uniform(prg);
    ct.body = q2.random_uniform(prg);
    Rlwe out = mod_switch_sym(q2, ct, q3);
    o["MOD_SWITCH_SYM_MASK_AT_Q3"] = coeffs(q3, out.mask);
    o["MOD_SWITCH_SYM_BODY_AT_Q3"] = coeffs(q3, out.body);
  } else if (name == "mod_switch_asym") {  // kat_mod_switch_asym
    Prg prg("layer3-kat-mod-switch-asym");
    Rlwe ct;
    ct.mask = q2.random_uniform(prg);
    ct.body = q2.random_uniform(prg);
    Poly m, b;
    mod_switch_asym(q2, ct, q3, q4, m, b);
    o["MOD_SWITCH_ASYM_MASK_AT_Q3"] = coeffs(q3, m);
    o["MOD_SWITCH_ASYM_BODY_AT_Q4"] = coeffs(q4, b);
  } else if (name == "gen_rsk") {  // kat_gen_rsk_first_sample / kat_gen_rsk_prg_order
    Prg prg("layer3-kat-gen-rsk-rsk");
    Poly s1 = keygen(q3, T, prg);
    Poly s2 = keygen(q3s, T, prg);
    std::vector<Rlev> rsk = gen_rsk(q3, s1, q3s, s2, BASE, DEPTH, T, prg);
    o["GEN_RSK_J0_L0_MASK"] = coeffs(q3s, rsk[0][0].mask);
    o["GEN_RSK_J0_L0_BODY"] = coeffs(q3s, rsk[0][0].body);
    std::vector<u64> ms, bs;
    for (auto& rl : rsk)
      for (auto& s : rl) {
        auto a = coeffs(q3s, s.mask), b = coeffs(q3s, s.body);
        ms.insert(ms.end(), a.begin(), a.end());
        bs.insert(bs.end(), b.begin(), b.end());
      }
    o["GEN_RSK_FULL_MASK_STREAM"] = ms;
    o["GEN_RSK_FULL_BODY_STREAM"] = bs;
  } else if (name == "ring_switch") {  // kat_ring_switch_apply
    Prg prg("layer3-kat-ring-switch");
    Poly s1 = keygen(q3, T, prg);
    Poly s2 = keygen(q3s, T, prg);
    std::vector<Rlev> rsk = gen_rsk(q3, s1, q3s, s2, BASE, DEPTH, T, prg);
    std::vector<u64> m(N1);
    for (int i = 0; i < N1; ++i) m[i] = i % 16;
    Rlwe ct = encrypt(q3, s1, encode(q3, 16, m), T, prg);
    std::vector<RlevEval> rske;
    for (auto& r : rsk) rske.push_back(rlev_to_eval(q3s, r));
    Rlwe out = ring_switch(q3, ct, q3s, rske, BASE);
    o["RING_SWITCH_OUT_MASK"] = coeffs(q3s, out.mask);
    o["RING_SWITCH_OUT_BODY"] = coeffs(q3s, out.body);
  } else if (name == "rekey") {  // kat_rekey_secret_key
    Prg prg("layer3-kat-rekey");
    Poly sk = keygen(q2, T, prg);
    o["REKEY_SK_Q3_COEFFS"] = coeffs(q3, rekey(q2, sk, q3));
  } else if (name == "decrypt_asym") {  // kat_decrypt_asymmetric_recovery
    Prg prg("layer3-kat-decrypt-asym");
    Poly s2 = keygen(q3s, T, prg);
    std::vector<u64> m(N2);
    for (int i = 0; i < N2; ++i) m[i] = (3 * i + 1) % 16;
    Rlwe ct = encrypt(q3s, s2, encode(q3s, 16, m), T, prg);
    Poly mm, bb;
    mod_switch_asym(q3s, ct, q3s, q4s, mm, bb);
    o["DECRYPT_ASYM_RECOVERED"] = decrypt_asymmetric(q3s, s2, mm, bb, 1ull << 12, 16);
    o["DECRYPT_ASYM_INPUT_PLAINTEXT"] = m;
  }
  return o;
}

// ---- crates/via-primitives/tests/layer4_kats.rs ---------------------------
static Outputs layer4(const std::string& name) {
  const int N = 64, DEPTH = 3, CK_DEPTH = 16;
  const u64 P = 2, BASE = 4, CK_BASE = 2, Q_SMALL = 4096;
  Ring R = Ring::single(N, 65537);
  Dist T = Dist::ternary();
  auto bit_poly = [&](u64 b) { return R.scalar_const(b); };
  auto enc = [&](std::vector<u64> c, const Poly& sk, Prg& prg) {
    c.resize(N, 0);
    return encrypt(R, sk, encode(R, P, c), T, prg);
  };
  auto rgsw_bit = [&](u64 b, const Poly& sk, Prg& prg) {
    return encrypt_rgsw(R, sk, bit_poly(b), BASE, BASE, DEPTH, DEPTH, T, prg);
  };
  Outputs o;
  auto put = [&](const std::string& k, const Rlwe& c) {
    o[k + "_MASK"] = coeffs(R, c.mask);
    o[k + "_BODY"] = coeffs(R, c.body);
  };
  if (name == "rotate") {
    Prg prg("layer4-kat-rotate");
    Poly sk = keygen(R, T, prg);
    put("ROTATE_K3", rotate(R, enc({1}, sk, prg), 3));
  } else if (name == "cmux") {
    Prg prg("layer4-kat-cmux");
    Poly sk = keygen(R, T, prg);
    Rgsw g = rgsw_bit(1, sk, prg);
    Rlwe c0 = enc({1}, sk, prg), c1 = enc({0, 1}, sk, prg);
    put("CMUX_SELECT1", cmux(R, rgsw_to_eval(R, g), c0, c1, BASE, BASE));
  } else if (name == "dmux") {
    Prg prg("layer4-kat-dmux");
    Poly sk = keygen(R, T, prg);
    Rgsw g = rgsw_bit(1, sk, prg);
    Rlwe c = enc({1, 1}, sk, prg), r0, r1;
    dmux(R, rgsw_to_eval(R, g), c, BASE, BASE, r0, r1);
    put("DMUX_BIT1_RESULT0", r0);
    put("DMUX_BIT1_RESULT1", r1);
  } else if (name == "cmux_tree") {
    Prg prg("layer4-kat-cmux-tree");
    Poly sk = keygen(R, T, prg);
    std::vector<RgswEval> bits;
    for (int i = 0; i < 2; ++i) bits.push_back(rgsw_to_eval(R, rgsw_bit(1, sk, prg)));
    std::vector<Rlwe> in;
    for (int i = 0; i < 4; ++i) {
      std::vector<u64> c(N, 0);
      c[i] = 1;
      in.push_back(encrypt(R, sk, encode(R, P, c), T, prg));
    }
    put("CMUX_TREE_IDX3", cmux_tree(R, bits, in, BASE, BASE));
  } else if (name == "dmux_tree") {
    Prg prg("layer4-kat-dmux-tree");
    Poly sk = keygen(R, T, prg);
    RgswEval b0 = rgsw_to_eval(R, rgsw_bit(1, sk, prg));
    RgswEval b1 = rgsw_to_eval(R, rgsw_bit(0, sk, prg));
    Rlwe c = enc({1, 1}, sk, prg);
    auto out = dmux_tree(R, {b0, b1}, c, BASE, BASE);
    for (int i = 0; i < 4; ++i) put("DMUX_TREE_IDX2_OUT" + std::to_string(i), out[i]);
  } else if (name == "crot_forward" || name == "crot_slot_extract") {
    bool fwd = name == "crot_forward";
    Prg prg(fwd ? "layer4-kat-crot-forward" : "layer4-kat-crot-slot-extract");
    Poly sk = keygen(R, T, prg);
    std::vector<RgswEval> bits;
    for (int i = 0; i < 2; ++i) bits.push_back(rgsw_to_eval(R, rgsw_bit(1, sk, prg)));
    Rlwe c = enc({1}, sk, prg);
    Rlwe out = crot(R, fwd ? CRotDir::Forward : CRotDir::SlotExtract, bits, c, BASE, BASE);
    put(fwd ? "CROT_FORWARD_ROT3" : "CROT_SLOT_EXTRACT_ROT3", out);
  } else if (name == "rlwe_to_rgsw") {
    Prg prg("layer4-kat-rlwe-to-rgsw");
    Poly sk = keygen(R, T, prg);
    Poly m = bit_poly(1);
    std::vector<u128> g = gadget_vector_values(R.Q(), BASE, DEPTH);
    std::vector<Rlwe> levels;
    for (int i = 0; i < DEPTH; ++i) levels.push_back(encrypt(R, sk, R.mul(m, R.scalar_const(g[i])), T, prg));
    Rlev ck = encrypt_rlev(R, sk, R.mul(sk, sk), CK_BASE, CK_DEPTH, T, prg);
    Rlev mrlev = encrypt_rlev(R, sk, m, BASE, DEPTH, T, prg);
    Rlwe cp = enc({1, 1}, sk, prg);
    Rgsw rg = rlwe_to_rgsw(R, levels, rlev_to_eval(R, ck), mrlev, CK_BASE);
    put("RLWE_TO_RGSW_NEG_S_M_L0", rg.neg_s_m[0]);
    put("RLWE_TO_RGSW_EXT_PRODUCT", external_product(R, rgsw_to_eval(R, rg), cp, BASE, BASE));
  } else if (name == "mod_switch_rgsw") {
    Prg prg("layer4-kat-mod-switch-rgsw");
    Poly sk = keygen(R, T, prg);
    Rgsw g = rgsw_bit(1, sk, prg);
    Ring Rs = Ring::single(N, Q_SMALL);
    Rgsw s = mod_switch_rgsw(R, g, Rs);
    o["MOD_SWITCH_RGSW_NEG_S_M_L0_MASK"] = coeffs(Rs, s.neg_s_m[0].mask);
    o["MOD_SWITCH_RGSW_NEG_S_M_L0_BODY"] = coeffs(Rs, s.neg_s_m[0].body);
    o["MOD_SWITCH_RGSW_M_L0_MASK"] = coeffs(Rs, s.m[0].mask);
    o["MOD_SWITCH_RGSW_M_L0_BODY"] = coeffs(Rs, s.m[0].body);
  }
  return o;
}

// ---- crates/via-primitives/tests/layer5_kats.rs ---------------------------
static Outputs layer5(const std::string& name) {
  const u64 Q = 65537, P = 16, BASE = 8, MESSAGE = 5;
  const int DEPTH = 6;
  Ring R8 = Ring::single(8, Q), R4 = Ring::single(4, Q);
  Dist T = Dist::ternary();
  Outputs o;
  auto lwe_out = [&](const Lwe& l) {
    o["ENCRYPT_LWE_MASKS"] = std::vector<u64>(l.mask_poly.begin(), l.mask_poly.end());
    o["ENCRYPT_LWE_BODY"] = {l.body[0]};
  };
  if (name == "embed_mlwe") {
    Prg kp("layer5-kat-embed-key");
    Poly sk = keygen(R4, T, kp);
    Prg ep("layer5-kat-embed-enc");
    Rlwe ct = encrypt(R4, sk, encode(R4, P, {1, 2, 3, 4}), T, ep);
    o["EMBED_MLWE_MASK0"] = embed_at(R4, ct.mask, 8, 0);
    o["EMBED_MLWE_BODY"] = embed_at(R4, ct.body, 8, 0);
  } else if (name == "encrypt_lwe") {
    Prg kp("layer5-kat-encrypt-lwe-key");
    Poly sk = keygen(R8, T, kp);
    Prg ep("layer5-kat-encrypt-lwe-enc");
    lwe_out(encrypt_lwe(R8, sk, MESSAGE, P, T, ep));
  } else if (name == "conv_d") {
    Prg kp("layer5-kat-conv-key");
    Poly sk = keygen(R8, T, kp);
    Prg ep("layer5-kat-conv-enc");
    Lwe lwe = encrypt_lwe(R8, sk, MESSAGE, P, T, ep);
    Prg gp("layer5-kat-conv-keygen");
    CascadeKey key = gen_cascade_key(R8, sk, BASE, DEPTH, T, gp);
    CascadeKeyEval ke = cascade_key_to_eval(R8, key);
    Mlwe in;
    for (int i = 0; i < 8; ++i) in.masks.push_back(Poly{lwe.mask_poly[i]});
    in.body = lwe.body;
    Mlwe out = conv_step(R8.with_n(2), R8.with_n(1), in, ke.steps[0], BASE);
    o["CONV_D_OUT_MASK0"] = out.masks[0];
    o["CONV_D_OUT_BODY"] = out.body;
  } else if (name == "gen_lwe_to_rlwe_key") {
    Prg kp("layer5-kat-keygen-key");
    Poly sk = keygen(R8, T, kp);
    Prg gp("layer5-kat-keygen-gen");
    CascadeKey key = gen_cascade_key(R8, sk, BASE, DEPTH, T, gp);
    o["LWE2RLWE_KEY_STEP0_S0_L0_MASK"] = key.steps[0][0][0].mask;
  } else if (name == "lwe_to_rlwe") {
    Prg kp("layer5-kat-cascade-key");
    Poly sk = keygen(R8, T, kp);
    Prg ep("layer5-kat-cascade-enc");
    Lwe lwe = encrypt_lwe(R8, sk, MESSAGE, P, T, ep);
    Prg gp("layer5-kat-cascade-keygen");
    CascadeKey key = gen_cascade_key(R8, sk, BASE, DEPTH, T, gp);
    Rlwe r = lwe_to_rlwe(R8, lwe, cascade_key_to_eval(R8, key), BASE);
    o["LWE2RLWE_OUT_MASK"] = r.mask;
    o["LWE2RLWE_OUT_BODY"] = r.body;
  }
  return o;
}

// ---- crates/via-integration/tests/layer6_kats.rs --------------------------
Params layer6_params() {
  Params p;
  p.n1 = 8;
  p.n2 = 4;
  p.n_rec = 4;
  p.num_rows = 2;
  p.num_cols = 2;
  p.q1_0 = 1ull << 36;
  p.q1_1 = 0;
  p.q2 = 1ull << 28;
  p.q3 = 1ull << 20;
  p.q4 = 1ull << 12;
  p.p = 16;
  p.b_dmux = 64;
  p.b_cmux = 64;
  p.ck_base = 64;
  p.b_rsk = 8;
  p.l_query = 7;
  p.l_ck = 7;
  p.l_rsk = 8;
  return p;
}

static Outputs layer6(const std::string& name) {
  Params prm = layer6_params();
  Dist T = Dist::ternary();
  Ring R1 = prm.r1();
  Outputs o;
  if (name == "encrypt_lwe_raw") {
    Prg kp("layer6-kat-elr-key");
    Poly sk = keygen(R1, T, kp);
    Prg ep("layer6-kat-elr-enc");
    Lwe l = encrypt_lwe_raw(R1, sk, (u128)0xDEADBEEFull % R1.Q(), T, ep);
    o["ENCRYPT_LWE_RAW_MASKS"] = l.mask_poly;
    o["ENCRYPT_LWE_RAW_BODY"] = l.body;
  } else if (name == "gen_rlwe_to_rgsw_key") {
    Prg kp("layer6-kat-ck-key");
    Poly sk = keygen(R1, T, kp);
    Prg gp("layer6-kat-ck-gen");
    Rlev k = encrypt_rlev(R1, sk, R1.mul(sk, sk), prm.ck_base, prm.l_ck, T, gp);
    o["RLWE_TO_RGSW_KEY_S0_MASK"] = k[0].mask;
    o["RLWE_TO_RGSW_KEY_S0_BODY"] = k[0].body;
  } else if (name == "query_comp") {
    Prg sp("layer6-kat-qc-setup");
    PublicKeys pk;
    Client c = client_setup(prm, T, T, T, sp, pk);
    Prg qp("layer6-kat-qc-query");
    std::vector<Lwe> q = client_query(c, 5, prm.d(), qp);
    std::vector<u64> ms, bs;
    for (auto& l : q) {
      ms.insert(ms.end(), l.mask_poly.begin(), l.mask_poly.end());
      bs.push_back(l.body[0]);
    }
    o["QUERY_COMP_MASKS"] = ms;
    o["QUERY_COMP_BODIES"] = bs;
  } else if (name == "resp_comp") {
    Ring R2 = prm.r2(), R3n1 = prm.r3n1(), R3 = prm.r3();
    Prg s1p("layer6-kat-rc-s1");
    Poly sk1 = keygen(R2, T, s1p);
    Prg s2p("layer6-kat-rc-s2");
    Poly sk2 = keygen(R3, T, s2p);
    Prg ep("layer6-kat-rc-enc");
    std::vector<u64> msg(8, 0);
    msg[0] = 3;
    Rlwe ct = encrypt(R2, sk1, encode(R2, prm.p, msg), T, ep);
    Poly s1q3 = rekey(R2, sk1, R3n1);
    Prg rp("layer6-kat-rc-rsk");
    std::vector<Rlev> rsk = gen_rsk(R3n1, s1q3, R3, sk2, prm.b_rsk, prm.l_rsk, T, rp);
    std::vector<RlevEval> rske;
    for (auto& r : rsk) rske.push_back(rlev_to_eval(R3, r));
    Poly m, b;
    resp_comp(prm, ct, rske, m, b);
    o["RESP_COMP_MASK_Q3"] = m;
    o["RESP_COMP_BODY_Q4"] = b;
  }
  return o;
}

// ---- PRG / sampler unit vectors (prim/sampling/{prg,ternary,uniform}.rs) ----
static Outputs sampling(const std::string& name) {
  Outputs o;
  auto bytes = [](const char* seed, size_t skip, size_t n) {
    Prg p(seed, strlen(seed));
    std::vector<u8> tmp(skip + n);
    if (skip) p.fill(tmp.data(), skip);
    p.fill(tmp.data() + skip, n);
    return std::vector<u64>(tmp.begin() + skip, tmp.end());
  };
  auto below = [](u64 bound, int n) {
    Prg p("test");
    std::vector<u64> v;
    for (int i = 0; i < n; ++i) v.push_back(p.uniform_below(bound));
    return v;
  };
  auto tern = [](const char* seed) {
    Prg p(seed, strlen(seed));
    std::vector<i64> s(16);
    sample_into(Dist::ternary(), p, s.data(), 16);
    return std::vector<u64>(s.begin(), s.end());  // two's complement
  };
  if (name == "prg") {
    o["EMPTY_SEED_FIRST_32"] = bytes("", 0, 32);
    o["TEST_SEED_FIRST_32"] = bytes("test", 0, 32);
    o["TEST_SEED_BOUNDARY_134_138"] = bytes("test", 134, 4);
    o["TEST_SEED_RANDBELOW_3_FIRST_8"] = below(3, 8);
    o["TEST_SEED_RANDBELOW_256_FIRST_8"] = below(256, 8);
    o["TEST_SEED_RANDBELOW_Q3_FIRST_4"] = below(8380417, 4);
    o["TEST_SEED_RANDBELOW_2P32_FIRST_4"] = below(1ull << 32, 4);
    o["TEST_SEED_RANDBELOW_2P32_PLUS_1_FIRST_4"] = below((1ull << 32) + 1, 4);
  } else if (name == "ternary") {
    o["TEST_SEED_TP_N16"] = tern("test");
    o["EMPTY_SEED_TP_N16"] = tern("");
  } else if (name == "uniform") {
    auto uz = [](u64 q, int n) {
      Prg p("test");
      std::vector<u64> v;
      for (int i = 0; i < n; ++i) v.push_back(p.uniform_below(q));
      return v;
    };
    o["TEST_SEED_UP_Q17_N16"] = uz(17, 16);
    o["TEST_SEED_UP_Q3_N8"] = uz(8380417, 8);
    o["TEST_SEED_UP_Q1_FACTOR_N6"] = uz(137438822401ull, 6);
  }
  return o;
}

Outputs run_kat(const std::string& layer, const std::string& scenario) {
  if (layer == "layer3") return layer3(scenario);
  if (layer == "layer4") return layer4(scenario);
  if (layer == "layer5") return layer5(scenario);
  if (layer == "layer6") return layer6(scenario);
  if (layer == "sampling") return sampling(scenario);
  throw OracleError(ERR_INVALID, "unknown KAT layer " + layer);
}

}  // namespace vo
