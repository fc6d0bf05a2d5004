// Primitive operations of the reference on caller device buffers: the
// negacyclic NTT (crates/via-primitives/src/algebra/ring/ntt.rs:305-399), the
// RGSW x RLWE external product (encryption/rgsw.rs:108-121) and the key switch
// (encryption/keyswitch.rs:99-102) composed with the monomial rotation
// X^k * ct (algebra/ring/element.rs:328). These are the operations the
// reference's own kernel benchmarks time; they run the same kernels as the
// answer path.
//
// A ring here is built with NTT tables for exactly its degree, so the root is
// the reference's (the primitive 2n-th root from the smallest base,
// ntt.rs:150-198) and eval-form outputs equal the reference's.
#include <map>
#include <memory>
#include <mutex>
#include <tuple>

#include "gadget.cuh"
#include "server.cuh"

namespace via {

void prim_external_products(const DevRing& R, const Gadget& g, const u64* rgsw, const u64* cts, long count, u64* out,
                            u64* rgsw_eval, u64* digits, cudaStream_t st);
void prim_key_switches(const DevRing& R, const Gadget& g, const u64* key, const u64* cts, const u64* shifts, long count,
                       u64* out, u64* key_eval, u64* masks, u64* bodies, u64* digits, u64* prod, cudaStream_t st);

namespace {

struct PrimRing {
  DevRing R;
  std::vector<NttTableHost> tables;
};

std::mutex g_mu;  // guards the ring cache and the scratch below
std::map<std::tuple<int, int, u64, u64>, std::unique_ptr<PrimRing>> g_rings;
std::map<int, std::unique_ptr<DevBuf>> g_scratch;  // per device, grow-only

struct ApiErr : std::runtime_error {
  via_status st;
  ApiErr(via_status s, const std::string& m) : std::runtime_error(m), st(s) {}
};

// The ring of `d` on the current device (built once; the caller holds g_mu).
const DevRing& prim_ring(const via_ring_desc* d) {
  if (!d) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null ring");
  const int n = (int)d->n;
  if (n < 2 || n > 4096 || (n & (n - 1))) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "ring degree must be a power of two in 2..4096");
  if (d->nl != 1 && d->nl != 2) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "ring limbs must be 1 or 2");
  const u64 q0 = d->q[0], q1 = d->nl == 2 ? d->q[1] : 0;
  for (int l = 0; l < (int)d->nl; ++l) {
    const u64 q = l ? q1 : q0;
    if (q >= (1ull << 50) || !is_ntt_friendly(q, n))
      throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "every prime must be below 2^50 and NTT-friendly at this degree");
  }
  if (q1 == q0) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "RNS primes must differ");
  int dev = 0;
  VIA_CUDA(cudaGetDevice(&dev));
  auto key = std::make_tuple(dev, n, q0, q1);
  auto it = g_rings.find(key);
  if (it != g_rings.end()) return it->second->R;
  std::unique_ptr<PrimRing> P(new PrimRing());
  DevRing& R = P->R;
  R.n = n;
  R.nl = (int)d->nl;
  R.m[0] = make_devmod(q0);
  R.m[1] = q1 ? make_devmod(q1) : R.m[0];
  if (q1) {
    R.q0inv_mod_q1 = h_inv(q0 % q1, q1);
    R.q0inv_shoup = (u64)(((u128)R.q0inv_mod_q1 << 64) / q1);
  }
  P->tables.reserve(2);
  for (int l = 0; l < R.nl; ++l) {
    P->tables.push_back(make_ntt_table(l ? q1 : q0, n));  // tables for exactly this degree
    if (!P->tables.back().valid) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "no NTT table for this prime");
    R.t[l] = P->tables.back().dev;
  }
  if (R.nl == 1) R.t[1] = R.t[0];
  R.ntt = true;
  const DevRing& out = P->R;
  g_rings[key] = std::move(P);
  return out;
}

u64* prim_scratch(size_t count) {
  int dev = 0;
  VIA_CUDA(cudaGetDevice(&dev));
  auto& b = g_scratch[dev];
  if (!b) b.reset(new DevBuf());
  if (b->n < count) {
    VIA_CUDA(cudaDeviceSynchronize());  // earlier calls may still read the old buffer
    b->alloc(count);
  }
  return b->p;
}

Gadget prim_gadget(const DevRing& R, u64 base, uint32_t L) {
  if (base < 2 || L < 1 || L > 64) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "gadget base must be >= 2 and 1 <= L <= 64");
  return make_gadget(base, (int)L, R);
}

template <class F>
via_status guarded_prim(F&& f) {
  try {
    f();
    set_last_error("");
    return VIA_OK;
  } catch (const ApiErr& e) {
    set_last_error(e.what());
    return e.st;
  } catch (const CudaError& e) {
    set_last_error(e.what());
    return e.status == 101 ? VIA_ERR_OUT_OF_MEMORY : e.status == 100 ? VIA_ERR_INVALID_ARGUMENT : VIA_ERR_CUDA;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return VIA_ERR_CUDA;
  }
}

}  // namespace
}  // namespace via

using namespace via;

extern "C" {

via_status via_ntt_forward_dev(const via_ring_desc* ring, uint64_t* data, uint64_t count, void* stream) {
  return guarded_prim([&] {
    if (!data || count == 0) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null data or empty batch");
    std::lock_guard<std::mutex> g(g_mu);
    const DevRing& R = prim_ring(ring);
    ntt_forward(data, R.n, R.nl, (long)count * R.nl, R.t[0], R.t[1], (cudaStream_t)stream);
  });
}

via_status via_ntt_inverse_dev(const via_ring_desc* ring, uint64_t* data, uint64_t count, void* stream) {
  return guarded_prim([&] {
    if (!data || count == 0) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null data or empty batch");
    std::lock_guard<std::mutex> g(g_mu);
    const DevRing& R = prim_ring(ring);
    ntt_inverse(data, R.n, R.nl, (long)count * R.nl, R.t[0], R.t[1], (cudaStream_t)stream);
  });
}

via_status via_external_product_dev(const via_ring_desc* ring, uint64_t base, uint32_t levels, const uint64_t* rgsw,
                                    const uint64_t* rlwe, uint64_t count, uint64_t* out, void* stream) {
  return guarded_prim([&] {
    if (!rgsw || !rlwe || !out || count == 0 || count > (1u << 24))
      throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null buffer or batch outside 1..2^24");
    std::lock_guard<std::mutex> g(g_mu);
    const DevRing& R = prim_ring(ring);
    const Gadget gd = prim_gadget(R, base, levels);
    const size_t per = (size_t)R.nl * R.n;
    const size_t ev = count * 2 * levels * 2 * per, dg = count * 2 * levels * per;
    u64* s = prim_scratch(ev + dg);
    cudaStream_t st = (cudaStream_t)stream;
    prim_external_products(R, gd, rgsw, rlwe, (long)count, out, s, s + ev, st);
    VIA_CUDA(cudaStreamSynchronize(st));  // the scratch is reused by the next call
  });
}

via_status via_key_switch_dev(const via_ring_desc* ring, uint64_t base, uint32_t levels, const uint64_t* key,
                              const uint64_t* rlwe, const uint64_t* shifts, uint64_t count, uint64_t* out,
                              void* stream) {
  return guarded_prim([&] {
    if (!key || !rlwe || !shifts || !out || count == 0 || count > (1u << 24))
      throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "null buffer or batch outside 1..2^24");
    std::lock_guard<std::mutex> g(g_mu);
    const DevRing& R = prim_ring(ring);
    const Gadget gd = prim_gadget(R, base, levels);
    const size_t per = (size_t)R.nl * R.n;
    const size_t ke = (size_t)levels * 2 * per, mk = count * per, dg = count * levels * per, pr = count * 2 * per;
    u64* s = prim_scratch(ke + 2 * mk + dg + pr);
    cudaStream_t st = (cudaStream_t)stream;
    prim_key_switches(R, gd, key, rlwe, shifts, (long)count, out, s, s + ke, s + ke + mk, s + ke + 2 * mk,
                      s + ke + 2 * mk + dg, st);
    VIA_CUDA(cudaStreamSynchronize(st));
  });
}

via_status via_gadget_digits_host(uint64_t q0, uint64_t q1, uint64_t base, uint32_t levels, const uint64_t* coeffs,
                                  uint64_t count, int64_t* out) {
  return guarded_prim([&] {
    if (!coeffs || !out || q0 < 2 || levels < 1 || levels > 64 || base < 2)
      throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "bad arguments");
    DevRing R;
    R.n = 1;
    R.nl = q1 ? 2 : 1;
    R.m[0] = make_devmod(q0);
    R.m[1] = q1 ? make_devmod(q1) : R.m[0];
    if (q1) {
      R.q0inv_mod_q1 = h_inv(q0 % q1, q1);
      if (!R.q0inv_mod_q1) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "RNS primes are not coprime");
      R.q0inv_shoup = (u64)(((u128)R.q0inv_mod_q1 << 64) / q1);
    }
    const Gadget g = make_gadget(base, (int)levels, R);
    i64 d[64];
    for (uint64_t i = 0; i < count; ++i) {
      const u64 a0 = coeffs[i * R.nl], a1 = R.nl == 2 ? coeffs[i * R.nl + 1] : 0;
      if (a0 >= q0 || (q1 && a1 >= q1)) throw ApiErr(VIA_ERR_INVALID_ARGUMENT, "residue out of range");
      decompose_coeff(a0, a1, R, g, d);
      for (uint32_t k = 0; k < levels; ++k) out[i * levels + k] = d[k];
    }
  });
}

}  // extern "C"
