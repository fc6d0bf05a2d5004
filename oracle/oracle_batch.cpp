// VIA-B on the CPU (test infrastructure only): Extr, the pair conversion, the
// repack engine with the cascade-key suffix switched to q2, and answer_batch.
//
//   crates/via-primitives/src/conversion/extract.rs:61-75      extr
//   crates/via-primitives/src/conversion/repack.rs:64-181      embed_d, mlwes_to_mlwe
//   crates/via-primitives/src/conversion/repack.rs:232-316     repack engine body
//   crates/via-primitives/src/conversion/repack.rs:650-739     q1 -> q2 key derivation
//   crates/via-server/src/batch.rs:72-163                      answer_batch
//   crates/via-client/src/batch.rs:35-58                       deinterleave_batch
#include <exception>
#include <mutex>
#include <thread>

#include "via_oracle.hpp"

namespace vo {

// Extr_g: an RLWE of degree n -> a (n/g, g)-MLWE. masks[0] = pi_0(A),
// masks[k] = pi_{r-k}(A) * X for k >= 1 (r = n/g), body = pi_0(B).
Mlwe extr(const Ring& R, const Rlwe& ct, int g) {
  const int rank = R.n / g;
  Ring Rg = R.with_n(g);
  Mlwe out;
  for (int k = 0; k < rank; ++k) {
    if (k == 0)
      out.masks.push_back(project_at(R, ct.mask, g, 0));
    else
      out.masks.push_back(Rg.mul_x_pow(project_at(R, ct.mask, g, rank - k), 1));
  }
  out.body = project_at(R, ct.body, g, 0);
  return out;
}

// embed_d with d = 2 (slots 0 and 1) followed by conv_step's key switches and
// slot reduction on the already-embedded masks.
Mlwe mlwes_to_mlwe(const Ring& Rout, const Ring& Rin, const Mlwe& a, const Mlwe& b, const std::vector<RlevEval>& keys,
                   u64 base) {
  const size_t rank_in = a.masks.size(), rank_out = rank_in / 2;
  if (b.masks.size() != rank_in || keys.size() != rank_in)
    throw OracleError(ERR_INVALID, "mlwes_to_mlwe: rank mismatch");
  auto embed2 = [&](const Poly& x, const Poly& y) {
    Poly r = embed_at(Rin, x, Rout.n, 0);
    Rout.add_inplace(r, embed_at(Rin, y, Rout.n, 1));
    return r;
  };
  Mlwe out;
  out.masks.assign(rank_out, Rout.zero());
  out.body = embed2(a.body, b.body);
  for (int group = 0; group < 2; ++group)
    for (size_t j = 0; j < rank_out; ++j) {
      const size_t idx = rank_out * group + j;
      Rlwe rl{embed2(a.masks[idx], b.masks[idx]), Rout.zero()};
      Rlwe sw = key_switch(Rout, keys[idx], rl, base);
      Rout.add_inplace(out.masks[j], sw.mask);
      Rout.add_inplace(out.body, sw.body);
    }
  return out;
}

// The repack step keys: the cascade steps whose output degree is 2*n3 .. n1,
// every RLev sample switched from q1 to q2 (mod_switch_sym) and put in eval form
// at q2. Entry s holds the keys of output degree 2*n3 << s.
std::vector<std::vector<RlevEval>> repack_keys(const Params& prm, const CascadeKey& ck) {
  Ring R1 = prm.r1(), R2 = prm.r2();
  std::vector<std::vector<RlevEval>> out;
  for (int nout = 2 * prm.n_rec; nout <= prm.n1; nout <<= 1) {
    int k = 0;
    while ((2 << k) != nout) ++k;  // steps[k] has output degree 2^(k+1)
    Ring Rs = R1.with_n(nout), Rd = R2.with_n(nout);
    std::vector<RlevEval> level;
    for (const Rlev& rl : ck.steps.at(k)) {
      Rlev sw;
      for (const Rlwe& smp : rl) sw.push_back(mod_switch_sym(Rs, smp, Rd));
      level.push_back(rlev_to_eval(Rd, sw));
    }
    out.push_back(std::move(level));
  }
  return out;
}

static size_t bit_reverse(size_t i, int bits) {
  size_t r = 0;
  for (int b = 0; b < bits; ++b) r = (r << 1) | ((i >> b) & 1);
  return r;
}

// Repack of T = n2 / n3 CRot outputs at (n1, q2): Extr_{n3} each into an
// (n1/n3, n3)-MLWE, bit-reverse the T inputs, pad with zero MLWEs to n1/n3,
// then log2(n1/n3) levels of pair conversion, and unwrap the rank-1 result.
Rlwe repack(const Params& prm, const std::vector<Rlwe>& rotated, const std::vector<std::vector<RlevEval>>& keys) {
  Ring R2 = prm.r2();
  const int g = prm.n_rec, D = prm.n1 / g;
  const size_t T = rotated.size();
  std::vector<Mlwe> v;
  for (size_t i = 0; i < T; ++i) v.push_back(extr(R2, rotated[i], g));
  int lt = 0;
  while (((size_t)1 << lt) < T) ++lt;
  for (size_t i = 0; i < T; ++i) {
    size_t j = bit_reverse(i, lt);
    if (i < j) std::swap(v[i], v[j]);
  }
  Ring Rg = R2.with_n(g);
  Mlwe zero;
  zero.masks.assign(D, Rg.zero());
  zero.body = Rg.zero();
  while (v.size() < (size_t)D) v.push_back(zero);
  int level = 0;
  for (int nin = g; nin < prm.n1; nin <<= 1, ++level) {
    Ring Rin = R2.with_n(nin), Rout = R2.with_n(2 * nin);
    std::vector<Mlwe> nxt;
    for (size_t p = 0; p + 1 < v.size(); p += 2)
      nxt.push_back(mlwes_to_mlwe(Rout, Rin, v[p], v[p + 1], keys.at(level), prm.ck_base));
    v.swap(nxt);
  }
  return Rlwe{v.at(0).masks.at(0), v.at(0).body};
}

void answer_batch(const Params& prm, const std::vector<std::vector<Lwe>>& queries, const PreparedKeys& k,
                  const std::vector<std::vector<RlevEval>>& rkeys, const PreparedDb& db, int threads, Poly& mask_q3,
                  Poly& body_q4) {
  const size_t T = (size_t)(prm.n2 / prm.n_rec);
  if (queries.size() != T) throw OracleError(ERR_DIM_MISMATCH, "answer_batch: batch.len() must equal T");
  // The reference runs the T prefixes one after another (batch.rs:134-145).
  // They are independent, so the checker spreads them over its threads (each
  // prefix then scans single-threaded); the results are the same.
  std::vector<Rlwe> rotated(T);
  if (threads > 1 && T > 1) {
    const size_t w = std::min((size_t)threads, T);
    std::exception_ptr err;
    std::mutex mu;
    std::vector<std::thread> ts;
    for (size_t t = 0; t < w; ++t)
      ts.emplace_back([&, t] {
        for (size_t i = t; i < T; i += w) {
          try {
            rotated[i] = answer_through_crot(prm, queries[i], k, db, 1);
          } catch (...) {
            std::lock_guard<std::mutex> g(mu);
            if (!err) err = std::current_exception();
            return;
          }
        }
      });
    for (auto& th : ts) th.join();
    if (err) std::rethrow_exception(err);
  } else {
    for (size_t i = 0; i < T; ++i) rotated[i] = answer_through_crot(prm, queries[i], k, db, threads);
  }
  Rlwe packed = repack(prm, rotated, rkeys);
  resp_comp(prm, packed, k.rsk, mask_q3, body_q4);
}

}  // namespace vo
