// The client side of VIA on the device (crates/via-client/src): query
// generation and answer recovery, for load generation at serving rates and for
// clients that hold many queries at once.
//
//   query   : Client::query (crates/via-client/src/query.rs:75-130). Index ->
//             (gamma, alpha, beta); DMux bits of alpha MSB-first, CMux bits of
//             beta LSB-first, CRot bits of gamma LSB-first, L_QUERY LWEs per
//             bit, LWE j of a bit encrypting bit * g_j with the gadget vector
//             g_j = round(q1 / B^(j+1)) (gadget.rs:73-91), base b_dmux for DMux
//             bits and b_cmux for the others. Each LWE is encrypt_lwe_raw
//             (crates/via-primitives/src/encryption/lwe.rs): mask coefficients
//             drawn uniform_below(q_l) in row-major order, limb 0 first, then
//             one error sample, body = <mask, s1> + e + m per limb.
//   recover : decrypt_asymmetric (encryption/rlwe.rs:187-240): mask (x) s2 at q3,
//             rescaled to q4 with rounding, subtracted from the body, decoded
//             to plaintext mod p (round(p * c / q4), c centred).
//
// The PRG stream of a query is sequential (rejection sampling): its SHAKE256
// blocks are computed in parallel beforehand, one warp walks it 32 draws at a
// time, and the inner products run one CTA per LWE.
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "gadget.cuh"
#include "prg.cuh"
#include "server.cuh"

namespace via {
namespace {

constexpr int MAX_SEED = 64;

struct Draw {
  u64 bound[3];  // limb 0, limb 1, error range
  u64 mask[3];
  int nbytes[3];
};

Draw make_draw(const via_params& p, u64 err_range) {
  Draw D{};
  const u64 b[3] = {p.q1_0, p.q1_1 ? p.q1_1 : p.q1_0, err_range};
  for (int i = 0; i < 3; ++i) {
    const int bits = 64 - __builtin_clzll(b[i]);
    D.bound[i] = b[i];
    D.nbytes[i] = (bits + 7) / 8;
    D.mask[i] = bits == 64 ? ~(u64)0 : (((u64)1 << bits) - 1);
  }
  return D;
}

// Stream blocks [q][nblk][17] of every query's seed.
__global__ void k_client_blocks(const uint8_t* __restrict__ seeds, int seed_len, int nq, int nblk,
                                u64* __restrict__ blocks) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long)nq * nblk) return;
  const int q = (int)(gid / nblk), b = (int)(gid % nblk);
  u64 out[RATE_LANES];
  prg_block(seeds + (size_t)q * seed_len, seed_len, (u64)b, out);
  u64* dst = blocks + gid * RATE_LANES;
#pragma unroll
  for (int l = 0; l < RATE_LANES; ++l) dst[l] = out[l];
}

// One warp per query walks its stream through uniform_below (prg.rs), writing
// every LWE's mask ([nl][n1], limb-major) into `out` and its error sample
// (centred) into errs[q][lwe]. err_kind 0: ternary (draw r in [0,3): 0, 1,
// -1); 1: bounded uniform (draw - bound).
//
// The draws of a query form one sequence (per LWE: n1 * nl mask draws, then
// its error draw). Each round the 32 lanes take the next 32 draws at the byte
// offsets they would have if none were rejected (a prefix sum of their byte
// counts); the draws before the first rejected one are final, and the next
// round restarts at the rejected draw, after its bytes. With primes near a
// power of two rejections are rare, so a round settles ~32 draws. A draw
// rejected 64 times in a row raises the error flag. Blocks past the
// precomputed nblk are computed on the fly.
__global__ void k_client_walk(const u64* __restrict__ blocks, const uint8_t* __restrict__ seeds, int seed_len, int nq,
                              int nblk, int n_lwe, int n1, int nl, u64 lwe_len, Draw D, int err_kind, i64 err_bound,
                              u64* __restrict__ out, i64* __restrict__ errs, int* __restrict__ err) {
  const int q = (int)((blockIdx.x * (long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (q >= nq) return;  // warp-uniform
  const u64* blk = blocks + (size_t)q * nblk * RATE_LANES;
  const uint8_t* seed = seeds + (size_t)q * seed_len;
  u64 extra[RATE_LANES];
  long extra_idx = -1;
  auto byte_at = [&](u64 p) -> unsigned {
    const long b = (long)(p / SHAKE_RATE);
    const int o = (int)(p % SHAKE_RATE);
    u64 lane_v;
    if (b < nblk) {
      lane_v = blk[(size_t)b * RATE_LANES + o / 8];
    } else {
      if (b != extra_idx) {
        prg_block(seed, seed_len, (u64)b, extra);
        extra_idx = b;
      }
      lane_v = extra[o / 8];
    }
    return (unsigned)((lane_v >> (8 * (o % 8))) & 0xFF);
  };
  const long per = (long)n1 * nl + 1;  // draws per LWE
  const long total = per * n_lwe;
  long base = 0;
  u64 pos = 0;
  int run = 0;  // consecutive rejections of the draw at `base`
  while (base < total) {
    const long i = base + lane;
    const bool valid = i < total;
    int which = 2, l = 0, k = 0, j = 0;
    if (valid) {
      j = (int)(i / per);
      const long r = i % per;
      if (r < (long)n1 * nl) {
        l = (int)(r % nl);
        k = (int)(r / nl);
        which = l;
      }
    }
    const int nb = valid ? D.nbytes[which] : 0;
    int incl = nb;  // inclusive prefix sum of the byte counts
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += v;
    }
    const u64 at = pos + (u64)(incl - nb);
    u64 x = 0;
    for (int b = 0; b < nb; ++b) x |= (u64)byte_at(at + b) << (8 * b);
    x &= D.mask[which];
    const bool reject = valid && x >= D.bound[which];
    const unsigned rej = __ballot_sync(0xffffffffu, reject);
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    const int first = rej ? __ffs(rej) - 1 : 32;  // lanes below `first` hold final draws
    if (valid && lane < first) {
      if (which < 2) {
        out[((size_t)q * n_lwe + j) * lwe_len + (size_t)l * n1 + k] = x;
      } else {
        errs[(size_t)q * n_lwe + j] = err_kind == 0 ? (x == 0 ? 0 : (x == 1 ? 1 : -1)) : (i64)x - err_bound;
      }
    }
    if (rej) {
      const int through = __shfl_sync(0xffffffffu, incl, first);  // bytes up to and including the rejected draw
      pos += (u64)through;
      base += first;
      run = first == 0 ? run + 1 : 1;
      if (run >= 64) {
        if (lane == 0) atomicExch(err, 1);
        return;
      }
    } else {
      const int nvalid = __popc(vmask);
      pos += (u64)__shfl_sync(0xffffffffu, incl, nvalid - 1);
      base += nvalid;
      run = 0;
    }
  }
}

// One CTA per (query, LWE): body_l = <mask_l, s1_l> + e + m_l (mod q1_l).
__global__ void __launch_bounds__(256) k_client_body(u64* __restrict__ out, const u64* __restrict__ sk1,
                                                     const i64* __restrict__ errs, const u64* __restrict__ msgs,
                                                     int n1, int nl, u64 lwe_len, DevMod m0, DevMod m1) {
  const long lw = blockIdx.x;  // q * n_lwe + j
  u64* lwe = out + (size_t)lw * lwe_len;
  __shared__ u64 part[2][256][2];
  for (int l = 0; l < nl; ++l) {
    Acc128 acc{0, 0};
    for (int i = threadIdx.x; i < n1; i += blockDim.x) mac128(acc, lwe[(size_t)l * n1 + i], sk1[(size_t)l * n1 + i]);
    part[l][threadIdx.x][0] = acc.lo;
    part[l][threadIdx.x][1] = acc.hi;
  }
  __syncthreads();
  if (threadIdx.x < nl) {
    const int l = threadIdx.x;
    const DevMod& m = l ? m1 : m0;
    u64 r = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) r = addmod(r, reduce128(part[l][t][1], part[l][t][0], m), m.q);
    const i64 e = errs[lw];
    const u64 ev = e >= 0 ? reduce64((u64)e, m) : (m.q - reduce64((u64)(-e), m)) % m.q;
    r = addmod(addmod(r, ev, m.q), msgs[(size_t)lw * nl + l], m.q);
    lwe[(size_t)nl * n1 + l] = r;
  }
}

// One CTA per answer, n2 threads: decrypt_asymmetric and decode.
__global__ void k_client_recover(const u64* __restrict__ masks, const u64* __restrict__ bodies,
                                 const u64* __restrict__ sk2, int n2, DevMod m3, u64 q4, u64 p,
                                 u64* __restrict__ out) {
  extern __shared__ u64 sh[];
  u64* a = sh;
  u64* s = sh + n2;
  const long c = blockIdx.x;
  for (int i = threadIdx.x; i < n2; i += blockDim.x) {
    a[i] = masks[(size_t)c * n2 + i];
    s[i] = sk2[i];
  }
  __syncthreads();
  const u64 q3 = m3.q;
  for (int t = threadIdx.x; t < n2; t += blockDim.x) {
    Acc128 pos{0, 0}, neg{0, 0};
    for (int i = 0; i <= t; ++i) mac128(pos, a[i], s[t - i]);
    for (int i = t + 1; i < n2; ++i) mac128(neg, a[i], s[n2 + t - i]);
    const u64 prod = submod(reduce128(pos.hi, pos.lo, m3), reduce128(neg.hi, neg.lo, m3), q3);
    // round(prod * q4 / q3) mod q4 (prod in [0, q3)).
    const u128 v = ((u128)prod * q4 + q3 / 2) / q3;
    const u64 sw = (u64)(v % q4);
    const u64 b = bodies[(size_t)c * n2 + t];
    const u64 noisy = b >= sw ? b - sw : b + (q4 - sw);
    const i128 cc = noisy <= q4 / 2 ? (i128)noisy : (i128)noisy - (i128)q4;
    const i128 num = (i128)p * cc + (i128)(q4 / 2);
    i128 r = num / (i128)q4;
    if (num % (i128)q4 < 0) r -= 1;  // div_euclid
    i128 mm = r % (i128)p;
    if (mm < 0) mm += p;
    out[(size_t)c * n2 + t] = (u64)mm;
  }
}

struct ApiErr : std::runtime_error {
  via_status code;
  ApiErr(via_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

int ceil_log2(u64 v) {
  int r = 0;
  while (((u64)1 << r) < v) ++r;
  return r;
}

std::vector<u128> gadget_values(u128 Q, u64 base, int L) {
  std::vector<u128> g(L);
  u128 div = 1;
  for (int i = 0; i < L; ++i) {
    div *= base;
    g[i] = (Q + div / 2) / div;
  }
  return g;
}

}  // namespace

struct Client {
  via_params prm{};
  int device = 0;
  cudaStream_t stream = nullptr;
  DevBuf sk1, sk2;
  int err_kind = 0;
  i64 err_bound = 1;
  ~Client() {
    if (stream) cudaStreamDestroy(stream);
  }
};

}  // namespace via

using namespace via;

struct via_client : via::Client {};

namespace {

template <class F>
via_status client_guarded(F&& f) {
  try {
    f();
    set_last_error("");
    return VIA_OK;
  } catch (const ApiErr& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const CudaError& e) {
    set_last_error(e.what());
    return e.status == 101 ? VIA_ERR_OUT_OF_MEMORY : e.status == 100 ? VIA_ERR_INVALID_ARGUMENT : VIA_ERR_CUDA;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return VIA_ERR_CUDA;
  }
}

// Queries for `count` indices into the device buffer d_out [count][n_lwe][lwe_len].
void make_queries(via_client* c, const uint64_t* indices, uint64_t count, const uint8_t* seeds, uint32_t seed_len,
                  u64* d_out, cudaStream_t st) {
  const via_params& p = c->prm;
  const u64 I = p.num_rows, J = p.num_cols, d = p.n1 / p.n_rec;
  const int nd = ceil_log2(I), nc = ceil_log2(J), nr = ceil_log2(d), L = (int)p.l_query;
  const int n_lwe = (nd + nc + nr) * L, nl = p.q1_1 ? 2 : 1, n1 = (int)p.n1;
  const u64 ll = lwe_len(p);
  const u128 Q = (u128)p.q1_0 * (p.q1_1 ? p.q1_1 : 1);
  const std::vector<u128> gd = gadget_values(Q, p.b_dmux, L), gc = gadget_values(Q, p.b_cmux, L);
  // Message residues per (query, LWE, limb).
  std::vector<u64> msgs((size_t)count * n_lwe * nl);
  for (u64 q = 0; q < count; ++q) {
    const u64 index = indices[q];
    if (index >= d * I * J)
      throw ApiErr(VIA_ERR_INDEX_OUT_OF_RANGE, "index " + std::to_string(index) + " out of range");
    const u64 group = I * J, gamma = index / group, alpha = (index % group) / J, beta = index % J;
    std::vector<std::pair<int, const std::vector<u128>*>> bits;
    for (int i = 0; i < nd; ++i) bits.push_back({(int)((alpha >> (nd - 1 - i)) & 1), &gd});
    for (int i = 0; i < nc; ++i) bits.push_back({(int)((beta >> i) & 1), &gc});
    for (int i = 0; i < nr; ++i) bits.push_back({(int)((gamma >> i) & 1), &gc});
    size_t j = 0;
    for (auto& b : bits)
      for (int k = 0; k < L; ++k, ++j) {
        const u128 m = b.first ? (*b.second)[k] % Q : 0;
        for (int l = 0; l < nl; ++l) msgs[((size_t)q * n_lwe + j) * nl + l] = (u64)(m % (l ? p.q1_1 : p.q1_0));
      }
  }
  const Draw D = make_draw(p, c->err_kind == 0 ? 3 : (u64)(2 * c->err_bound + 1));
  // Every draw accepted, plus 2% and two blocks for rejections (more are made on the fly).
  const u64 per_lwe = (u64)n1 * (D.nbytes[0] + (nl == 2 ? D.nbytes[1] : 0)) + D.nbytes[2];
  const u64 need = per_lwe * n_lwe;
  const int nblk = (int)((need + need / 50) / SHAKE_RATE + 2);
  DevBuf d_seeds(((size_t)count * seed_len + 7) / 8), d_blocks((size_t)count * nblk * RATE_LANES),
      d_errs((size_t)count * n_lwe), d_msgs(msgs.size()), d_flag(1);
  VIA_CUDA(cudaMemsetAsync(d_flag.p, 0, 8, st));
  VIA_CUDA(cudaMemcpyAsync(d_seeds.p, seeds, (size_t)count * seed_len, cudaMemcpyHostToDevice, st));
  VIA_CUDA(cudaMemcpyAsync(d_msgs.p, msgs.data(), msgs.size() * 8, cudaMemcpyHostToDevice, st));
  const long nb = (long)count * nblk;
  k_client_blocks<<<(unsigned)((nb + 127) / 128), 128, 0, st>>>(reinterpret_cast<const uint8_t*>(d_seeds.p),
                                                                (int)seed_len, (int)count, nblk, d_blocks.p);
  VIA_LAUNCHED();
  k_client_walk<<<(unsigned)((count + 3) / 4), 128, 0, st>>>(
      d_blocks.p, reinterpret_cast<const uint8_t*>(d_seeds.p), (int)seed_len, (int)count, nblk, n_lwe, n1, nl, ll, D,
      c->err_kind, c->err_bound, d_out, reinterpret_cast<i64*>(d_errs.p), reinterpret_cast<int*>(d_flag.p));
  VIA_LAUNCHED();
  const DevMod m0 = make_devmod(p.q1_0), m1 = make_devmod(p.q1_1 ? p.q1_1 : p.q1_0);
  k_client_body<<<(unsigned)(count * n_lwe), 256, 0, st>>>(d_out, c->sk1.p, reinterpret_cast<const i64*>(d_errs.p),
                                                           d_msgs.p, n1, nl, ll, m0, m1);
  VIA_LAUNCHED();
  int flag = 0;
  VIA_CUDA(cudaMemcpyAsync(&flag, d_flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  VIA_CUDA(cudaStreamSynchronize(st));  // the temporaries are freed on return
  if (flag) throw ApiErr(VIA_ERR_INVALID_PRG_SEED, "client query: a PRG stream rejected 64 draws in a row");
}

void check_client_args(via_client* c, const uint64_t* indices, uint64_t count, const uint8_t* seeds,
                       uint32_t seed_len) {
  if (!c || !indices || !seeds || count == 0 || count > (1u << 20))
    throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null argument or count outside 1..2^20");
  if (seed_len == 0 || seed_len > MAX_SEED) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "seed_len must be in 1..64");
}

}  // namespace

extern "C" {

via_status via_client_create(const via_params* params, const uint64_t* sk1, const uint64_t* sk2, uint32_t err_kind,
                             uint32_t err_bound, via_client** out) {
  return client_guarded([&] {
    if (!params || !sk1 || !sk2 || !out) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (err_kind > 1 || (err_kind == 1 && (err_bound == 0 || err_bound > (1u << 30))))
      throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "error distribution: kind 0 (ternary) or 1 (bounded uniform, bound >= 1)");
    validate_params(*params);
    std::unique_ptr<via_client> c(new via_client());
    c->prm = *params;
    c->err_kind = (int)err_kind;
    c->err_bound = err_kind == 1 ? (i64)err_bound : 1;
    VIA_CUDA(cudaGetDevice(&c->device));
    VIA_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    const int nl = params->q1_1 ? 2 : 1;
    c->sk1.alloc((size_t)nl * params->n1);
    c->sk2.alloc(params->n2);
    VIA_CUDA(cudaMemcpy(c->sk1.p, sk1, c->sk1.n * 8, cudaMemcpyHostToDevice));
    VIA_CUDA(cudaMemcpy(c->sk2.p, sk2, c->sk2.n * 8, cudaMemcpyHostToDevice));
    *out = c.release();
  });
}

void via_client_destroy(via_client* c) { delete c; }

via_status via_client_queries(via_client* c, const uint64_t* indices, uint64_t count, const uint8_t* seeds,
                              uint32_t seed_len, uint64_t* out) {
  return client_guarded([&] {
    check_client_args(c, indices, count, seeds, seed_len);
    if (!out) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null output");
    const size_t len = (size_t)count * query_lwes(c->prm) * lwe_len(c->prm);
    DevBuf d(len);
    make_queries(c, indices, count, seeds, seed_len, d.p, c->stream);
    VIA_CUDA(cudaMemcpyAsync(out, d.p, len * 8, cudaMemcpyDeviceToHost, c->stream));
    VIA_CUDA(cudaStreamSynchronize(c->stream));
  });
}

via_status via_client_queries_dev(via_client* c, const uint64_t* indices, uint64_t count, const uint8_t* seeds,
                                  uint32_t seed_len, uint64_t* out, void* stream) {
  return client_guarded([&] {
    check_client_args(c, indices, count, seeds, seed_len);
    if (!out) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null output");
    make_queries(c, indices, count, seeds, seed_len, out, stream ? (cudaStream_t)stream : c->stream);
  });
}

via_status via_client_recover(via_client* c, const uint64_t* masks, const uint64_t* bodies, uint64_t count,
                              uint64_t* out) {
  return client_guarded([&] {
    if (!c || !masks || !bodies || !out || count == 0 || count > (1u << 20))
      throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null argument or count outside 1..2^20");
    const via_params& p = c->prm;
    const size_t len = (size_t)count * p.n2;
    DevBuf dm(len), db(len), dout(len);
    VIA_CUDA(cudaMemcpyAsync(dm.p, masks, len * 8, cudaMemcpyHostToDevice, c->stream));
    VIA_CUDA(cudaMemcpyAsync(db.p, bodies, len * 8, cudaMemcpyHostToDevice, c->stream));
    const int threads = (int)std::min<u64>(p.n2, 1024);
    k_client_recover<<<(unsigned)count, threads, 2 * p.n2 * 8, c->stream>>>(dm.p, db.p, c->sk2.p, (int)p.n2,
                                                                            make_devmod(p.q3), p.q4, p.p, dout.p);
    VIA_LAUNCHED();
    VIA_CUDA(cudaMemcpyAsync(out, dout.p, len * 8, cudaMemcpyDeviceToHost, c->stream));
    VIA_CUDA(cudaStreamSynchronize(c->stream));
  });
}

}  // extern "C"
