// Query wire formats (crates/via-protocol/src/wire/format.rs:93-190) and the
// device-side mask regeneration of the PRG-compressed format.
//
// A query on the wire is n_lwe packets, one per LWE ciphertext, each starting
// with the format tag of format.rs:
//   0x00 Uncompressed : [0x00][count: u64 LE][count u64 LE]   count = nl * (n1 + 1)
//                       (the LWE verbatim: mask polynomial limb-major, then body)
//   0x01 PrgCompressed: [0x01][seed: 32 bytes][count: u64 LE][count u64 LE]   count = nl
//                       (the body verbatim; the mask is regenerated)
// Mask regeneration (format.rs:20-27,146-160): Shake256Prg(seed), then
// uniform_below(q_l) for every mask coefficient in row-major order, one draw
// per limb, limb 0 first (prim/sampling/prg.rs:108-206). The PRG's byte stream
// is counter-mode, block b = SHAKE256(seed || le64(b))[0..136), so every block
// is one Keccak-f[1600] permutation and the device computes all blocks of all
// packets in parallel; one thread per packet then walks its stream through the
// rejection sampler (an accepted draw consumes ceil(bitlen(q) / 8) bytes).
#include <cstring>
#include <string>
#include <vector>

#include "prg.cuh"
#include "server.cuh"

namespace via {
namespace {

constexpr int SEED_LEN = 32;

// All PRG blocks of all compressed packets: blocks [pkt][nblk][17].
__global__ void k_prg_blocks(const uint8_t* __restrict__ seeds, int npkt, int nblk, u64* __restrict__ blocks) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long)npkt * nblk) return;
  const int pkt = (int)(gid / nblk), b = (int)(gid % nblk);
  u64 out[RATE_LANES];
  prg_block(seeds + (size_t)pkt * SEED_LEN, SEED_LEN, (u64)b, out);
  u64* dst = blocks + gid * RATE_LANES;
#pragma unroll
  for (int l = 0; l < RATE_LANES; ++l) dst[l] = out[l];
}

struct Sampler {
  u64 q[2];
  u64 mask[2];
  int nbytes[2];
};

// One thread per compressed packet: uniform_below over the packet's stream,
// writing the mask polynomial of LWE lwe[pkt] ([nl][n1] limb-major) of `query`.
// Blocks beyond the precomputed nblk (a run of rejections) are computed here.
__global__ void k_prg_masks(const u64* __restrict__ blocks, const uint8_t* __restrict__ seeds,
                            const int* __restrict__ lwe, int npkt, int nblk, int n1, int nl, u64 lwe_len, Sampler S,
                            u64* __restrict__ query, int* __restrict__ err) {
  const int pkt = blockIdx.x * blockDim.x + threadIdx.x;
  if (pkt >= npkt) return;
  const u64* blk = blocks + (size_t)pkt * nblk * RATE_LANES;
  u64 extra[RATE_LANES];
  long extra_idx = -1;
  u64 pos = 0;  // byte position in the stream
  auto byte_at = [&](u64 p) -> unsigned {
    const long b = (long)(p / SHAKE_RATE);
    const int o = (int)(p % SHAKE_RATE);
    u64 lane;
    if (b < nblk) {
      lane = blk[(size_t)b * RATE_LANES + o / 8];
    } else {
      if (b != extra_idx) {
        prg_block(seeds + (size_t)pkt * SEED_LEN, SEED_LEN, (u64)b, extra);
        extra_idx = b;
      }
      lane = extra[o / 8];
    }
    return (unsigned)((lane >> (8 * (o % 8))) & 0xFF);
  };
  u64* out = query + (size_t)lwe[pkt] * lwe_len;
  for (int k = 0; k < n1; ++k)
    for (int l = 0; l < nl; ++l) {
      // q >= 2^(bits-1) accepts at least half of the draws, so 64 rejections in
      // a row (probability below 2^-64) end the packet with an error instead.
      u64 v = 0;
      bool ok = false;
      for (int attempt = 0; attempt < 64 && !ok; ++attempt) {
        v = 0;
        for (int b = 0; b < S.nbytes[l]; ++b) v |= (u64)byte_at(pos + b) << (8 * b);
        pos += S.nbytes[l];
        v &= S.mask[l];
        ok = v < S.q[l];
      }
      if (!ok) {
        atomicExch(err, 1);
        return;
      }
      out[(size_t)l * n1 + k] = v;
    }
}

struct ApiErr : std::runtime_error {
  via_status code;
  ApiErr(via_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

u64 rd64(const uint8_t* p) {
  u64 v = 0;
  for (int i = 0; i < 8; ++i) v |= (u64)p[i] << (8 * i);
  return v;
}

// Parses the packets into `query` (host, flat layout); compressed packets
// leave their mask to the device and are listed in seeds / lwes.
void parse_wire(const via_params& p, const uint8_t* wire, u64 len, u64* query, std::vector<uint8_t>& seeds,
                std::vector<int>& lwes) {
  const u64 n_lwe = query_lwes(p), ll = lwe_len(p), nl = p.q1_1 ? 2 : 1;
  u64 off = 0;
  for (u64 w = 0; w < n_lwe; ++w) {
    if (off >= len) throw ApiErr(VIA_ERR_BUFFER_TOO_SHORT, "wire query: " + std::to_string(w) + " of " +
                                                               std::to_string(n_lwe) + " LWE packets present");
    const uint8_t tag = wire[off];
    u64* dst = query + w * ll;
    if (tag == 0x00) {
      if (len - off < 9) throw ApiErr(VIA_ERR_BUFFER_TOO_SHORT, "wire query: truncated packet header");
      const u64 count = rd64(wire + off + 1);
      if (count != ll) throw ApiErr(VIA_ERR_DIM_MISMATCH, "wire query: uncompressed LWE length mismatch");
      if ((len - off - 9) / 8 < count) throw ApiErr(VIA_ERR_BUFFER_TOO_SHORT, "wire query: truncated LWE");
      for (u64 i = 0; i < count; ++i) dst[i] = rd64(wire + off + 9 + 8 * i);
      off += 9 + 8 * count;
    } else if (tag == 0x01) {
      if (len - off < 1 + SEED_LEN + 8) throw ApiErr(VIA_ERR_BUFFER_TOO_SHORT, "wire query: truncated packet header");
      const u64 count = rd64(wire + off + 1 + SEED_LEN);
      if (count != nl) throw ApiErr(VIA_ERR_DIM_MISMATCH, "wire query: compressed body length mismatch");
      if ((len - off - 1 - SEED_LEN - 8) / 8 < count) throw ApiErr(VIA_ERR_BUFFER_TOO_SHORT, "wire query: truncated body");
      seeds.insert(seeds.end(), wire + off + 1, wire + off + 1 + SEED_LEN);
      lwes.push_back((int)w);
      std::memset(dst, 0, (size_t)ll * 8);
      for (u64 i = 0; i < count; ++i) dst[nl * p.n1 + i] = rd64(wire + off + 1 + SEED_LEN + 8 + 8 * i);
      off += 1 + SEED_LEN + 8 + 8 * count;
    } else {
      throw ApiErr(VIA_ERR_UNKNOWN_FORMAT_TAG, "wire query: unknown format tag " + std::to_string(tag));
    }
  }
  if (off != len) throw ApiErr(VIA_ERR_QUERY_LENGTH_MISMATCH, "wire query: bytes after the last of " +
                                                                  std::to_string(n_lwe) + " LWE packets");
}

Sampler make_sampler(const via_params& p) {
  Sampler S{};
  const u64 qs[2] = {p.q1_0, p.q1_1 ? p.q1_1 : p.q1_0};
  for (int l = 0; l < 2; ++l) {
    const int bits = 64 - __builtin_clzll(qs[l]);
    S.q[l] = qs[l];
    S.nbytes[l] = (bits + 7) / 8;
    S.mask[l] = bits == 64 ? ~(u64)0 : (((u64)1 << bits) - 1);
  }
  return S;
}

// Decodes a wire query into the device buffer d_query (flat layout).
void decode_to_device(Server& s, const uint8_t* wire, u64 len, u64* d_query, cudaStream_t st) {
  const via_params& p = s.prm;
  const u64 n_lwe = query_lwes(p), ll = lwe_len(p);
  const int nl = p.q1_1 ? 2 : 1;
  std::vector<u64> host(n_lwe * ll);
  std::vector<uint8_t> seeds;
  std::vector<int> lwes;
  parse_wire(p, wire, len, host.data(), seeds, lwes);
  VIA_CUDA(cudaMemcpyAsync(d_query, host.data(), host.size() * 8, cudaMemcpyHostToDevice, st));
  const int npkt = (int)lwes.size();
  if (npkt) {
    const Sampler S = make_sampler(p);
    const int nbytes = std::max(S.nbytes[0], S.nbytes[1]);
    // Every draw accepted: n1 * nl draws; 1% and 2 blocks of margin for rejections
    // (more are generated on the fly).
    const u64 need = (u64)p.n1 * nl * nbytes;
    const int nblk = (int)((need + need / 100) / SHAKE_RATE + 2);
    DevBuf d_seeds((seeds.size() + 7) / 8), d_lwes((lwes.size() + 1) / 2), d_blocks((size_t)npkt * nblk * RATE_LANES),
        d_err(1);
    VIA_CUDA(cudaMemsetAsync(d_err.p, 0, 8, st));
    VIA_CUDA(cudaMemcpyAsync(d_seeds.p, seeds.data(), seeds.size(), cudaMemcpyHostToDevice, st));
    VIA_CUDA(cudaMemcpyAsync(d_lwes.p, lwes.data(), lwes.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    const long nb = (long)npkt * nblk;
    k_prg_blocks<<<(unsigned)((nb + 127) / 128), 128, 0, st>>>(reinterpret_cast<const uint8_t*>(d_seeds.p), npkt, nblk,
                                                               d_blocks.p);
    VIA_LAUNCHED();
    k_prg_masks<<<(unsigned)((npkt + 63) / 64), 64, 0, st>>>(d_blocks.p, reinterpret_cast<const uint8_t*>(d_seeds.p),
                                                            reinterpret_cast<const int*>(d_lwes.p), npkt, nblk, p.n1, nl,
                                                            ll, S, d_query, reinterpret_cast<int*>(d_err.p));
    VIA_LAUNCHED();
    int err = 0;
    VIA_CUDA(cudaMemcpyAsync(&err, d_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    VIA_CUDA(cudaStreamSynchronize(st));  // the temporaries are freed on return
    if (err) throw ApiErr(VIA_ERR_INVALID_PRG_SEED, "wire query: a PRG seed's stream rejected 64 draws in a row");
  }
}

template <class F>
via_status wire_guarded(F&& f) {
  try {
    f();
    return VIA_OK;
  } catch (const ApiErr& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const CudaError& e) {
    set_last_error(e.what());
    return e.status == 101 ? VIA_ERR_OUT_OF_MEMORY : VIA_ERR_CUDA;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return VIA_ERR_INVALID_ARGUMENT;
  }
}

}  // namespace

}  // namespace via

using namespace via;

extern "C" {

via_status via_query_from_wire(via_server* s, const uint8_t* wire, uint64_t len, uint64_t* out_query,
                               uint64_t out_len) {
  return wire_guarded([&] {
    if (!s || !wire || !out_query) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null argument");
    const via_params& p = s->prm;
    const u64 total = query_lwes(p) * lwe_len(p);
    if (out_len < total) throw ApiErr(VIA_ERR_BUFFER_TOO_SHORT, "output shorter than one query");
    DevBuf d(total);
    decode_to_device(*s, wire, len, d.p, s->stream);
    VIA_CUDA(cudaMemcpyAsync(out_query, d.p, total * 8, cudaMemcpyDeviceToHost, s->stream));
    VIA_CUDA(cudaStreamSynchronize(s->stream));
  });
}

via_status via_server_answer_wire(via_server* s, const uint8_t* wire, uint64_t len, uint64_t* out_mask,
                                  uint64_t* out_body) {
  return wire_guarded([&] {
    if (!s || !wire || !out_mask || !out_body) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null argument");
    if (!s->cascade_eval.p) throw ApiErr(VIA_ERR_SETUP_NOT_COMPLETE, "server has no public keys");
    const via_params& p = s->prm;
    std::lock_guard<std::mutex> g(s->mu);
    decode_to_device(*s, wire, len, workspace_query(*s), s->stream);
    answer_graph(*s, 1, s->stream);
    VIA_CUDA(cudaMemcpyAsync(out_mask, workspace_answer_mask(*s), p.n2 * 8, cudaMemcpyDeviceToHost, s->stream));
    VIA_CUDA(cudaMemcpyAsync(out_body, workspace_answer_body(*s), p.n2 * 8, cudaMemcpyDeviceToHost, s->stream));
    VIA_CUDA(cudaStreamSynchronize(s->stream));
  });
}

}  // extern "C"
