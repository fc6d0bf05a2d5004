// Server::setup / answer / destroy behind the C ABI of include/via_gpu.h.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "first_dim.cuh"
#include "server.cuh"

namespace via {

struct ApiError : std::runtime_error {
  via_status code;
  ApiError(via_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

unsigned long long g_kernel_launches = 0;
static thread_local std::string g_last_error;

// Scratch for via_first_dim_scan_static: the split selection vectors (five
// byte planes padded to 16 rows per query and row, 16 * I * n1 bytes) live in
// this file-scope device array instead of memory the call allocates. Every
// device that loads the library holds it (8 MiB) until exit.
// bytes: 16 * I_pad * n1 <= 2^23 with I_pad = num_rows rounded up to 64 (I_pad <= 256 at n1 = 2048)
constexpr u64 STATIC_SCAN_SCRATCH = 8ull << 20;
static __device__ __align__(256) uint4 g_scan_scratch[STATIC_SCAN_SCRATCH / 16];
// Device address of g_scan_scratch per device, resolved once with that device current.
static std::mutex g_scan_scratch_mu;
static uint8_t* g_scan_scratch_addr[128] = {nullptr};

void set_last_error(const std::string& m) { g_last_error = m; }

template <class F>
static via_status guarded(F&& f) {
  try {
    f();
    g_last_error.clear();
    return VIA_OK;
  } catch (const ApiError& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const CudaError& e) {
    g_last_error = e.what();
    return e.status == 101 ? VIA_ERR_OUT_OF_MEMORY : (e.status == 100 ? VIA_ERR_INVALID_ARGUMENT : VIA_ERR_CUDA);
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return VIA_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return VIA_ERR_INVALID_ARGUMENT;
  }
}

void DevBuf::alloc(size_t count) {
  free();
  if (count == 0) return;
  cudaError_t e = cudaMalloc(&p, count * 8);
  if (e != cudaSuccess) {
    p = nullptr;
    (void)cudaGetLastError();
    throw CudaError(101, "cudaMalloc(" + std::to_string(count * 8) + " bytes): " + cudaGetErrorString(e));
  }
  n = count;
}
void DevBuf::free() {
  if (p) cudaFree(p);
  p = nullptr;
  n = 0;
}

// Raises VIA_ERR_TIMEOUT once the FirstDim scan has reported that one of its
// bounded waits ran out (the word stays set for the handle's lifetime).
static void check_device_flags(Server& s, cudaStream_t st) {
  if (!s.fd_err.p) return;
  int flag = 0;
  VIA_CUDA(cudaMemcpyAsync(&flag, s.fd_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  VIA_CUDA(cudaStreamSynchronize(st));
  if (flag)
    throw ApiError(VIA_ERR_TIMEOUT, "FirstDim scan: a bounded device wait ran out (flag " + std::to_string(flag) + ")");
}

int ilog2(u64 v) { return v <= 1 ? 0 : 63 - __builtin_clzll(v); }
static bool pow2(u64 v) { return v && !(v & (v - 1)); }

// Shape guards of Server::setup / answer_through_crot (srv/answer.rs:132-157,461-471).
void validate_params(const via_params& p) {
  if (!pow2(p.num_rows) || !pow2(p.num_cols))
    throw ApiError(VIA_ERR_DIM_MISMATCH, "num_rows and num_cols must be powers of two");
  if (!pow2(p.n1) || !pow2(p.n2) || !pow2(p.n_rec) || p.n2 > p.n1 || p.n_rec > p.n2 || p.n1 > 4096)
    throw ApiError(VIA_ERR_DIM_MISMATCH, "ring degrees must be powers of two with n_rec <= n2 <= n1 <= 4096");
  if (p.l_query == 0 || p.l_ck == 0 || p.l_rsk == 0 || p.l_query > 64 || p.l_ck > 64 || p.l_rsk > 64)
    throw ApiError(VIA_ERR_INVALID_ARGUMENT, "gadget depths must be in 1..64");
  for (u64 b : {p.b_dmux, p.b_cmux, p.ck_base, p.b_rsk})
    if (b < 2 || b >= (1ull << 32)) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "gadget bases must be in [2, 2^32)");
  for (u64 q : {p.q1_0, p.q2, p.q3, p.q4, p.p})
    if (q < 2 || q >= (1ull << 62)) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "moduli must be in [2, 2^62)");
  if (p.q1_1 && (p.q1_1 < 2 || p.q1_1 >= (1ull << 62)))
    throw ApiError(VIA_ERR_INVALID_ARGUMENT, "moduli must be in [2, 2^62)");
  if (p.p > p.q4 || p.q4 > p.q3) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "moduli must satisfy p <= q4 <= q3");
}

u64 lwe_len(const via_params& p) { return (u64)(p.q1_1 ? 2 : 1) * (p.n1 + 1); }
u64 query_lwes(const via_params& p) {
  u64 d3 = p.n1 / p.n_rec;
  return (u64)(ilog2(p.num_rows) + ilog2(p.num_cols) + (d3 > 1 ? ilog2(d3) : 0)) * p.l_query;
}
u64 cascade_key_len(const via_params& p) {
  return (u64)ilog2(p.n1) * 2 * p.n1 * p.l_ck * 2 * (p.q1_1 ? 2 : 1);
}
u64 conv_key_len(const via_params& p) { return (u64)p.l_ck * 2 * (p.q1_1 ? 2 : 1) * p.n1; }
u64 rsk_len(const via_params& p) { return (u64)(p.n1 / p.n2) * p.l_rsk * 2 * p.n2; }

u64 h_inv(u64 a, u64 m) {
  i128 t = 0, nt = 1, r = m, nr = a % m;
  while (nr) {
    i128 qq = r / nr, tmp = t - qq * nt;
    t = nt;
    nt = tmp;
    tmp = r - qq * nr;
    r = nr;
    nr = tmp;
  }
  if (r != 1) return 0;
  return (u64)(t < 0 ? t + m : t);
}

static DevRing make_ring(Server& s, int n, u64 q0, u64 q1) {
  DevRing R;
  R.n = n;
  R.nl = q1 ? 2 : 1;
  R.m[0] = make_devmod(q0);
  if (q1) {
    R.m[1] = make_devmod(q1);
    R.q0inv_mod_q1 = h_inv(q0 % q1, q1);
    if (!R.q0inv_mod_q1) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "q1 RNS primes are not coprime");
    R.q0inv_shoup = (u64)(((u128)R.q0inv_mod_q1 << 64) / q1);
  } else {
    R.m[1] = R.m[0];
  }
  // Lazy 128-bit multiply-accumulates need T * q^2 < 2^128 for T <= 256 terms.
  bool ok = q0 < (1ull << 50) && q1 < (1ull << 50) && is_ntt_friendly(q0, n) && (!q1 || is_ntt_friendly(q1, n));
  if (ok) {
    for (int l = 0; l < R.nl; ++l) {
      u64 q = l ? q1 : q0;
      // Reuse a table of this prime when one with nmax >= n exists.
      const NttTable* found = nullptr;
      for (auto& t : s.tables)
        if (t.valid && t.dev.q == q && t.dev.nmax >= n) found = &t.dev;
      if (!found) {
        int nmax = n;
        while (nmax < 4096 && is_ntt_friendly(q, nmax * 2)) nmax *= 2;
        s.tables.push_back(make_ntt_table(q, nmax));
        found = &s.tables.back().dev;
      }
      R.t[l] = *found;
    }
    if (R.nl == 1) R.t[1] = R.t[0];
    R.ntt = true;
  }
  return R;
}

// setup_db (srv/setup_db.rs:39-75) for one record slot k: record k*I*J + r
// lands in cell r at coefficient positions d*c + k, lifted p -> q2 unchanged.
__global__ void k_encode_slot(const void* __restrict__ recs, int fmt, u64 count, u64 r0, int k, int n1, int d,
                              int n_rec, u64 p, u64* __restrict__ db) {
  u64 gid = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= count * (u64)n_rec) return;
  u64 r = gid / n_rec;
  int c = (int)(gid % n_rec);
  u64 v;
  if (fmt == VIA_RECORDS_U64) {
    v = ((const u64*)recs)[gid];
  } else {
    unsigned char b = ((const unsigned char*)recs)[gid >> 1];
    v = (c & 1) ? (b >> 4) : (b & 15);
  }
  v = (p & (p - 1)) == 0 ? (v & (p - 1)) : v % p;
  db[(r0 + r) * (u64)n1 + (u64)d * c + k] = v;
}

Server::~Server() {
  workspace_destroy(*this);
  for (auto& t : tables) free_ntt_table(t);
  if (stream) cudaStreamDestroy(stream);
}

__global__ void k_u64_to_f64(const u64* __restrict__ in, double* __restrict__ out, long count) {
  const long gid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid < count) out[gid] = __ull2double_rn(in[gid]);
}

static void transform_keys(Server& s) {
  const via_params& p = s.prm;
  // Cascade: step k (output degree 2^k) has 2*n1*L_CK*2*nl residues.
  if (s.r1.ntt) {
    u64 step = (u64)2 * p.n1 * p.l_ck * 2 * s.r1.nl;
    for (int k = 1, nout = 2; nout <= (int)p.n1; ++k, nout <<= 1)
      ntt_forward(s.cascade_eval.p + (k - 1) * step, nout, s.r1.nl, (long)(step / nout), s.r1.t[0], s.r1.t[1],
                  s.stream);
    ntt_forward(s.conv_eval.p, p.n1, s.r1.nl, (long)p.l_ck * 2 * s.r1.nl, s.r1.t[0], s.r1.t[1], s.stream);
    if (ntt_fp_ok(s.r1.t[0], s.r1.t[1]) && p.ck_base <= 255) {  // the 8-bit digit path's double-precision MAC
      s.cascade_eval_d.alloc(s.cascade_eval.n);
      const long count = (long)s.cascade_eval.n;
      k_u64_to_f64<<<(unsigned)((count + 255) / 256), 256, 0, s.stream>>>(
          s.cascade_eval.p, reinterpret_cast<double*>(s.cascade_eval_d.p), count);
      VIA_LAUNCHED();
    }
  }
  if (s.r3.ntt)
    ntt_forward(s.rsk_eval.p, p.n2, 1, (long)(p.n1 / p.n2) * p.l_rsk * 2, s.r3.t[0], s.r3.t[1], s.stream);
}

static void load_keys(Server& s, const via_public_keys* keys) {
  if (!keys) return;
  const via_params& p = s.prm;
  if (!keys->cascade_key || !keys->conv_key || !keys->rsk) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null key buffer");
  s.cascade_eval.alloc(cascade_key_len(p));
  s.conv_eval.alloc(conv_key_len(p));
  s.rsk_eval.alloc(rsk_len(p));
  VIA_CUDA(cudaMemcpyAsync(s.cascade_eval.p, keys->cascade_key, s.cascade_eval.n * 8, cudaMemcpyHostToDevice, s.stream));
  VIA_CUDA(cudaMemcpyAsync(s.conv_eval.p, keys->conv_key, s.conv_eval.n * 8, cudaMemcpyHostToDevice, s.stream));
  VIA_CUDA(cudaMemcpyAsync(s.rsk_eval.p, keys->rsk, s.rsk_eval.n * 8, cudaMemcpyHostToDevice, s.stream));
  derive_repack_keys(s);  // VIA-B: from the coefficient-form cascade key, before it is transformed
  transform_keys(s);
}

static void setup(Server& s, const via_params& p, const via_public_keys* keys, const void* records, u64 n_records,
                  via_record_format fmt) {
  validate_params(p);
  s.prm = p;
  if (fmt != VIA_RECORDS_U64 && fmt != VIA_RECORDS_NIBBLE) throw ApiError(VIA_ERR_UNKNOWN_FORMAT_TAG, "unknown record format");
  if (fmt == VIA_RECORDS_NIBBLE && (p.p > 16 || p.n_rec % 2)) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "nibble records need p <= 16");
  u64 I = p.num_rows, J = p.num_cols;
  int d = (int)(p.n1 / p.n_rec);
  if (n_records > I * J * (u64)d)
    throw ApiError(VIA_ERR_DIM_MISMATCH, "setup: more records than DB capacity (would silently drop)");
  if (n_records && !records) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "records is null");
  VIA_CUDA(cudaGetDevice(&s.device));
  VIA_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
  s.r1 = make_ring(s, p.n1, p.q1_0, p.q1_1);
  s.r2 = make_ring(s, p.n1, p.q2, 0);
  s.r3n1 = make_ring(s, p.n1, p.q3, 0);
  s.r3 = make_ring(s, p.n2, p.q3, 0);
  s.r4 = make_ring(s, p.n2, p.q4, 0);

  // Prepared database (setup_db.rs:39-75, prepared_db.rs:57-85): records are
  // encoded into cells, lifted p -> q2 and transformed, 16 rows at a time.
  size_t rec_bytes = fmt == VIA_RECORDS_U64 ? (size_t)p.n_rec * 8 : (size_t)p.n_rec / 2;
  if (s.r2.ntt && !fd_supported((int)I, (int)p.n1, p.q2))
    throw ApiError(VIA_ERR_INVALID_ARGUMENT, "FirstDim needs num_rows <= 4096 and q2 < 2^40 for NTT-friendly q2");
  const bool tensor = s.r2.ntt;
  const u64 rows_per_pass = tensor ? 16 : I;
  DevBuf cells;  // u64 cells of one pass: [rows_per_pass][J][n1]
  if (tensor) {
    s.fd.I = (int)I;
    s.fd.J = (int)J;
    s.fd.n = (int)p.n1;
    s.fd.I_pad = fd_round_up((int)I, FD_KC);
    s.fd.J_pad = fd_round_up((int)J, FD_MT);
    s.fd.m = s.r2.m[0];
    s.fd.packed4 = fd_packable(p.q2);
    VIA_CUDA(cudaDeviceGetAttribute(&s.fd.grid, cudaDevAttrMultiProcessorCount, s.device));
    s.fd.smem_max = fd_prepare_device();
    s.planes = std::make_shared<DevBuf>();
    s.planes->alloc(fd_planes_bytes((int)I, (int)J, (int)p.n1, s.fd.packed4) / 8);
    VIA_CUDA(cudaMemsetAsync(s.planes->p, 0, s.planes->n * 8, s.stream));
    s.fd_err.alloc(1);
    VIA_CUDA(cudaMemsetAsync(s.fd_err.p, 0, 8, s.stream));
    s.fd.err = reinterpret_cast<int*>(s.fd_err.p);
    cells.alloc(rows_per_pass * J * p.n1);
  } else {
    s.db = std::make_shared<DevBuf>();
    s.db->alloc(I * J * p.n1);
  }
  u64* cell_buf = tensor ? cells.p : s.db->p;
  void* stage = nullptr;
  if (n_records) VIA_CUDA(cudaMalloc(&stage, (size_t)std::min<u64>(rows_per_pass * J, n_records) * rec_bytes));
  try {
    for (u64 i0 = 0; i0 < I; i0 += rows_per_pass) {
      const u64 rows = std::min<u64>(rows_per_pass, I - i0);
      VIA_CUDA(cudaMemsetAsync(cell_buf, 0, rows_per_pass * J * p.n1 * 8, s.stream));
      for (int k = 0; k < d; ++k) {
        // Records of slot k whose cells lie in rows [i0, i0 + rows).
        const u64 lo = (u64)k * I * J + i0 * J;
        const u64 hi = std::min<u64>(n_records, lo + rows * J);
        if (lo >= hi) continue;
        const char* src = (const char*)records + (size_t)lo * rec_bytes;
        VIA_CUDA(cudaMemcpyAsync(stage, src, (size_t)(hi - lo) * rec_bytes, cudaMemcpyHostToDevice, s.stream));
        u64 threads = (hi - lo) * p.n_rec;
        k_encode_slot<<<(unsigned)((threads + 255) / 256), 256, 0, s.stream>>>(stage, fmt, hi - lo, 0, k, p.n1, d,
                                                                               p.n_rec, p.p, cell_buf);
        VIA_LAUNCHED();
        VIA_CUDA(cudaStreamSynchronize(s.stream));
      }
      if (s.r2.ntt) ntt_forward(cell_buf, p.n1, 1, (long)(rows * J), s.r2.t[0], s.r2.t[0], s.stream);
      if (tensor) {
        s.fd.planes = reinterpret_cast<const uint8_t*>(s.planes->p);
        fd_rows_to_planes(cell_buf, (int)i0, s.fd, reinterpret_cast<uint8_t*>(s.planes->p), s.stream);
      }
    }
  } catch (...) {
    cudaFree(stage);
    throw;
  }
  if (stage) cudaFree(stage);
  VIA_CUDA(cudaStreamSynchronize(s.stream));
  cells.free();

  load_keys(s, keys);
  workspace_create(s, 1);
  VIA_CUDA(cudaStreamSynchronize(s.stream));
}

// A second handle over the prepared database of `base` with record degree
// n_rec: the cells (and their planes) are shared, not copied. Only n_rec may
// differ from the base's parameters; the view's record r = k*I*J + i*J + j is
// coefficients d*c + k (d = n1 / n_rec) of cell (i, j), as setup_db lays out
// records of that degree (setup_db.rs:39-75).
static void setup_view(Server& s, const Server& base, uint32_t n_rec, const via_public_keys* keys) {
  via_params p = base.prm;
  p.n_rec = n_rec;
  validate_params(p);
  s.prm = p;
  VIA_CUDA(cudaGetDevice(&s.device));
  if (s.device != base.device) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "a view must be made on its database's device");
  VIA_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
  s.r1 = make_ring(s, p.n1, p.q1_0, p.q1_1);
  s.r2 = make_ring(s, p.n1, p.q2, 0);
  s.r3n1 = make_ring(s, p.n1, p.q3, 0);
  s.r3 = make_ring(s, p.n2, p.q3, 0);
  s.r4 = make_ring(s, p.n2, p.q4, 0);
  s.db = base.db;
  s.planes = base.planes;
  s.fd = base.fd;  // geometry, device limits and tuned tiles
  if (s.planes) {
    s.fd_err.alloc(1);
    VIA_CUDA(cudaMemsetAsync(s.fd_err.p, 0, 8, s.stream));
    s.fd.err = reinterpret_cast<int*>(s.fd_err.p);
  }
  load_keys(s, keys);
  workspace_create(s, 1);
  VIA_CUDA(cudaStreamSynchronize(s.stream));
}

}  // namespace via

using namespace via;

extern "C" {

const char* via_last_error(void) { return g_last_error.c_str(); }

uint64_t via_lwe_len(const via_params* p) { return p ? lwe_len(*p) : 0; }
uint64_t via_query_len(const via_params* p) { return p ? query_lwes(*p) : 0; }
uint64_t via_cascade_key_len(const via_params* p) { return p ? cascade_key_len(*p) : 0; }
uint64_t via_conv_key_len(const via_params* p) { return p ? conv_key_len(*p) : 0; }
uint64_t via_rsk_len(const via_params* p) { return p ? rsk_len(*p) : 0; }

via_status via_server_setup(const via_params* params, const via_public_keys* keys, const void* records,
                            uint64_t n_records, via_record_format format, via_server** out) {
  return guarded([&] {
    if (!params || !out) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::unique_ptr<via_server> s(new via_server());
    setup(*s, *params, keys, records, n_records, format);
    *out = s.release();
  });
}

via_status via_server_view(via_server* base, uint32_t n_rec, const via_public_keys* keys, via_server** out) {
  return guarded([&] {
    if (!base || !out) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    std::unique_ptr<via_server> s(new via_server());
    setup_view(*s, *base, n_rec, keys);
    *out = s.release();
  });
}

void via_server_destroy(via_server* s) { delete s; }

via_status via_first_dim_dev(via_server* s, const uint64_t* switched, uint64_t* out, void* stream) {
  return guarded([&] {
    if (!s || !switched || !out) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const via_params& p = s->prm;
    DevBuf sel(2 * p.num_rows * p.n1);
    VIA_CUDA(cudaMemcpyAsync(sel.p, switched, sel.n * 8, cudaMemcpyDeviceToDevice, st));
    if (s->r2.ntt) ntt_forward(sel.p, p.n1, 1, (long)(2 * p.num_rows), s->r2.t[0], s->r2.t[0], st);
    std::lock_guard<std::mutex> g(s->mu);
    first_dim_queries(*s, sel.p, out, 1, workspace_sel_bytes(*s), st);
    if (s->r2.ntt) ntt_inverse(out, p.n1, 1, (long)(2 * p.num_cols), s->r2.t[0], s->r2.t[0], st);
    VIA_CUDA(cudaStreamSynchronize(st));
    check_device_flags(*s, st);
  });
}

via_status via_server_answer_dev(via_server* s, const uint64_t* query, uint64_t n_lwe, uint64_t* out_mask,
                                 uint64_t* out_body, void* stream) {
  return guarded([&] {
    if (!s || !query || !out_mask || !out_body) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument");
    u64 expected = query_lwes(s->prm);
    if (n_lwe != expected)
      throw ApiError(VIA_ERR_QUERY_LENGTH_MISMATCH, "query length mismatch: expected " + std::to_string(expected) +
                                                        " ciphertexts, got " + std::to_string(n_lwe));
    if (!s->cascade_eval.p) throw ApiError(VIA_ERR_SETUP_NOT_COMPLETE, "server has no public keys");
    const via_params& p = s->prm;
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> g(s->mu);
    VIA_CUDA(cudaMemcpyAsync(workspace_query(*s), query, n_lwe * lwe_len(p) * 8, cudaMemcpyDeviceToDevice, st));
    answer_graph(*s, 1, st);
    VIA_CUDA(cudaMemcpyAsync(out_mask, workspace_answer_mask(*s), p.n2 * 8, cudaMemcpyDeviceToDevice, st));
    VIA_CUDA(cudaMemcpyAsync(out_body, workspace_answer_body(*s), p.n2 * 8, cudaMemcpyDeviceToDevice, st));
  });
}

via_status via_first_dim_scan_dev(via_server* s, const uint64_t* sel_eval, uint64_t* out_eval, void* stream) {
  return guarded([&] {
    if (!s || !sel_eval || !out_eval) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> g(s->mu);
    first_dim_queries(*s, sel_eval, out_eval, 1, workspace_sel_bytes(*s), (cudaStream_t)stream);
  });
}

via_status via_server_transform_q2_dev(via_server* s, uint64_t* data, uint64_t count, int inverse, void* stream) {
  return guarded([&] {
    if (!s || (!data && count)) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument");
    if (count > (1ull << 31)) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "too many polynomials");
    if (!s->r2.ntt || count == 0) return;
    cudaStream_t st = (cudaStream_t)stream;
    if (inverse)
      ntt_inverse(data, s->prm.n1, 1, (long)count, s->r2.t[0], s->r2.t[0], st);
    else
      ntt_forward(data, s->prm.n1, 1, (long)count, s->r2.t[0], s->r2.t[0], st);
  });
}

via_status via_first_dim_scan_many_dev(via_server* s, const uint64_t* sel_eval, uint64_t n_queries,
                                       uint64_t* out_eval, void* stream) {
  return guarded([&] {
    if (!s || !sel_eval || !out_eval || n_queries == 0 || n_queries > 4096)
      throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument or batch size outside 1..4096");
    DevBuf scratch;
    if (s->tensor_fd()) scratch.alloc((fd_sel_bytes(s->fd, (int)n_queries) + 7) / 8);
    std::lock_guard<std::mutex> g(s->mu);
    first_dim_queries(*s, sel_eval, out_eval, (int)n_queries, reinterpret_cast<uint8_t*>(scratch.p),
                      (cudaStream_t)stream);
    VIA_CUDA(cudaStreamSynchronize((cudaStream_t)stream));  // scratch is freed on return
  });
}

// The FirstDim scan for callers that cannot allocate device memory: same kernel
// and result as via_first_dim_scan_dev, but its split-selection scratch is the
// static array above, so this call makes no allocation. The first call on a
// device resolves the array's device address (cudaGetSymbolAddress); make that
// first call before any stream capture. Every call shares the array: calls
// whose work overlaps on the GPU race on it. Each call writes every scratch byte
// that reaches its result (the padding rows it leaves alone only feed
// accumulator columns that are never read), so nothing has to start at zero.
// Like via_first_dim_scan_dev it returns once the scan is enqueued, so a scan
// whose bounded waits ran out is reported by the handle's next synchronous call.
via_status via_first_dim_scan_static(via_server* s, const uint64_t* sel_eval, uint64_t* out_eval, void* stream) {
  return guarded([&] {
    if (!s || !sel_eval || !out_eval) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument");
    const u64 need = s->tensor_fd() ? fd_sel_bytes(s->fd, 1) : 0;
    if (need > STATIC_SCAN_SCRATCH)
      throw ApiError(VIA_ERR_INVALID_ARGUMENT, "via_first_dim_scan_static: the split selection needs " +
                                                   std::to_string(need) + " bytes (16 * I_pad * n1, I_pad = num_rows "
                                                   "rounded up to 64), more than the static scratch of " +
                                                   std::to_string(STATIC_SCAN_SCRATCH) + " bytes");
    int dev = 0;
    VIA_CUDA(cudaGetDevice(&dev));
    if (dev != s->device)
      throw ApiError(VIA_ERR_INVALID_ARGUMENT, "via_first_dim_scan_static: the current device (" +
                                                   std::to_string(dev) + ") is not the server's device (" +
                                                   std::to_string(s->device) + ")");
    if (dev < 0 || dev >= 128) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    std::lock_guard<std::mutex> g(s->mu);  // fd.tuned may be re-sorted by the autotuner
    uint8_t* scratch = nullptr;
    {
      std::lock_guard<std::mutex> g(g_scan_scratch_mu);
      if (!g_scan_scratch_addr[dev]) {
        void* addr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&addr, g_scan_scratch);
        if (e != cudaSuccess)
          throw CudaError(102, std::string("cudaGetSymbolAddress(g_scan_scratch): ") + cudaGetErrorString(e));
        g_scan_scratch_addr[dev] = static_cast<uint8_t*>(addr);
      }
      scratch = g_scan_scratch_addr[dev];
    }
    first_dim_queries(*s, sel_eval, out_eval, 1, scratch, (cudaStream_t)stream);
  });
}

via_status via_debug_stage(via_server* s, const uint64_t* query, uint64_t n_lwe, int stage, uint64_t* out,
                           uint64_t out_len) {
  return guarded([&] {
    if (!s || !query || !out) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument");
    if (stage < 1 || stage > 7) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "stage must be in 1..7");
    const via_params& p = s->prm;
    if (n_lwe != query_lwes(p)) throw ApiError(VIA_ERR_QUERY_LENGTH_MISMATCH, "query length mismatch");
    u64 nl = p.q1_1 ? 2 : 1, nb = query_lwes(p) / p.l_query;
    u64 sizes[8] = {0, n_lwe * 2 * nl * p.n1, nb * 2 * p.l_query * 2 * nl * p.n1, p.num_rows * 2 * nl * p.n1,
                    p.num_rows * 2 * p.n1, p.num_cols * 2 * p.n1, 2 * (u64)p.n1, 2 * (u64)p.n1};
    if (out_len < sizes[stage]) throw ApiError(VIA_ERR_BUFFER_TOO_SHORT, "debug buffer too short");
    std::lock_guard<std::mutex> g(s->mu);
    DevBuf dq(n_lwe * lwe_len(p)), dm(p.n2), db(p.n2), dout(sizes[stage]);
    VIA_CUDA(cudaMemcpyAsync(dq.p, query, dq.n * 8, cudaMemcpyHostToDevice, s->stream));
    answer_device_stages(*s, dq.p, 1, dm.p, db.p, s->stream, stage, dout.p);
    VIA_CUDA(cudaMemcpyAsync(out, dout.p, sizes[stage] * 8, cudaMemcpyDeviceToHost, s->stream));
    VIA_CUDA(cudaStreamSynchronize(s->stream));
    check_device_flags(*s, s->stream);
  });
}

// Grows the workspace (and drops cached graphs) when a batch exceeds it.
static void ensure_batch(via_server* s, u64 nq) {
  if ((int)nq <= workspace_batch(*s)) return;
  VIA_CUDA(cudaStreamSynchronize(s->stream));
  workspace_destroy(*s);
  workspace_create(*s, (int)nq);
}

via_status via_server_reserve(via_server* s, uint64_t max_queries) {
  return guarded([&] {
    if (!s || max_queries == 0 || max_queries > 4096) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "bad batch size");
    std::lock_guard<std::mutex> g(s->mu);
    ensure_batch(s, max_queries);
  });
}

}  // extern "C"

namespace via {
// ---------------------------------------------------------------------------
// Scan autotuner: measures every candidate tile of the FirstDim scan for the
// given batch sizes on this server's database and keeps the fastest. A cache
// file (one line per measured configuration, keyed by device name, ring degree,
// grid and modulus) lets later processes skip the measurement.
namespace {

std::string tune_key(const Server& s, int nq) {
  cudaDeviceProp prop{};
  VIA_CUDA(cudaGetDeviceProperties(&prop, s.device));
  std::string dev = prop.name;
  for (char& c : dev)
    if (c == ' ' || c == '\t') c = '_';
  return "fd_tc/2 " + dev + " n=" + std::to_string(s.fd.n) + " I=" + std::to_string(s.fd.I) +
         " J=" + std::to_string(s.fd.J) + " q=" + std::to_string(s.fd.m.q) + " nq=" + std::to_string(nq);
}

struct CachedTile {
  FdTile tile;
  float ms = 0.f, default_ms = 0.f;
};

// Cache line: <key> | <n_max> <stages> <order> <ms> <default_ms>
std::vector<std::pair<std::string, CachedTile>> read_tune_cache(const char* path) {
  std::vector<std::pair<std::string, CachedTile>> out;
  if (!path || !*path) return out;
  FILE* f = fopen(path, "r");
  if (!f) return out;
  char line[512];
  while (fgets(line, sizeof line, f)) {
    char* bar = strchr(line, '|');
    if (!bar) continue;
    std::string key(line, bar - line);
    while (!key.empty() && key.back() == ' ') key.pop_back();
    CachedTile c;
    if (sscanf(bar + 1, "%d %d %d %f %f", &c.tile.n_max, &c.tile.stages, &c.tile.order, &c.ms, &c.default_ms) == 5)
      out.push_back({key, c});
  }
  fclose(f);
  return out;
}

void append_tune_cache(const char* path, const std::string& key, const CachedTile& c) {
  if (!path || !*path) return;
  FILE* f = fopen(path, "a");
  if (!f) throw ApiError(VIA_ERR_INVALID_ARGUMENT, std::string("cannot append to the tuning cache ") + path);
  fprintf(f, "%s | %d %d %d %.6f %.6f\n", key.c_str(), c.tile.n_max, c.tile.stages, c.tile.order, c.ms, c.default_ms);
  fclose(f);
}

via_scan_tile to_abi(const FdTile& t) { return via_scan_tile{(uint32_t)t.n_max, (uint32_t)t.stages, (uint32_t)t.order, 0}; }
FdTile from_abi(const via_scan_tile& t) { return FdTile{(int)t.n_max, (int)t.stages, (int)t.order}; }

}  // namespace

void autotune_scan(Server& s, Workspace& w, const std::vector<int>& sizes, const char* cache_path,
                   std::vector<via_scan_tuning>* out) {
  std::unique_lock<std::shared_mutex> plan(s.plan_mu);
  if (!s.tensor_fd()) {  // schoolbook rings have no tiles
    if (out)
      for (int nq : sizes) out->push_back(via_scan_tuning{(uint32_t)nq, {0, 0, 0, 0}, 0.f, 0.f, 0, 0});
    return;
  }
  const auto cache = read_tune_cache(cache_path);
  for (int nq : sizes) {
    const std::string key = tune_key(s, nq);
    const CachedTile* hit = nullptr;
    for (const auto& e : cache)
      if (e.first == key && fd_tile_valid(s.fd, nq, e.second.tile)) hit = &e.second;
    CachedTile best;
    uint32_t measured = 0;
    if (hit) {
      best = *hit;
    } else {
      // Two passes over the candidates, each kept at its faster pass: a
      // candidate timed during a clock or power dip is not chosen or lost on
      // one noisy measurement.
      std::vector<FdTuneResult> r = workspace_measure_tiles(s, w, nq, 3);
      const std::vector<FdTuneResult> r2 = workspace_measure_tiles(s, w, nq, 3);
      for (size_t i = 0; i < r.size() && i < r2.size(); ++i) r[i].ms = std::min(r[i].ms, r2[i].ms);
      check_device_flags(s, s.stream);
      best.tile = r[0].tile;
      best.ms = r[0].ms;
      best.default_ms = r[0].ms;
      for (const FdTuneResult& x : r)
        if (x.ms < best.ms) {
          best.tile = x.tile;
          best.ms = x.ms;
        }
      measured = (uint32_t)r.size();
      append_tune_cache(cache_path, key, best);
    }
    fd_set_tile(s.fd, nq, best.tile);
    if (out) out->push_back(via_scan_tuning{(uint32_t)nq, to_abi(best.tile), best.ms, best.default_ms, measured, 0});
  }
  ++s.plan_gen;
}

}  // namespace via

extern "C" {

via_status via_server_autotune(via_server* s, const uint32_t* batch_sizes, uint64_t count, const char* cache_path,
                               via_scan_tuning* out) {
  return guarded([&] {
    if (!s || !batch_sizes || count == 0 || count > 64)
      throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument or batch list outside 1..64 entries");
    std::vector<int> sizes;
    uint32_t bmax = 0;
    for (uint64_t i = 0; i < count; ++i) {
      if (batch_sizes[i] == 0 || batch_sizes[i] > 4096)
        throw ApiError(VIA_ERR_INVALID_ARGUMENT, "batch size outside 1..4096");
      bmax = std::max(bmax, batch_sizes[i]);
      sizes.push_back((int)batch_sizes[i]);
    }
    std::lock_guard<std::mutex> g(s->mu);
    if (s->tensor_fd()) ensure_batch(s, bmax);
    std::vector<via_scan_tuning> res;
    autotune_scan(*s, *s->ws, sizes, cache_path, &res);
    if (out)
      for (size_t i = 0; i < res.size(); ++i) out[i] = res[i];
  });
}

via_status via_server_set_scan_tile(via_server* s, uint32_t batch, const via_scan_tile* tile) {
  return guarded([&] {
    if (!s || batch == 0 || batch > 4096) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null handle or bad batch size");
    std::lock_guard<std::mutex> g(s->mu);
    std::unique_lock<std::shared_mutex> plan(s->plan_mu);  // service workers read fd.tuned under plan_mu
    if (!s->tensor_fd()) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "this server's scan has no tiles (schoolbook ring)");
    if (!tile) {
      auto& v = s->fd.tuned;
      v.erase(std::remove_if(v.begin(), v.end(), [&](const std::pair<int, FdTile>& e) { return e.first == (int)batch; }),
              v.end());
    } else {
      const FdTile t = from_abi(*tile);
      if (!fd_tile_valid(s->fd, (int)batch, t)) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "tile not valid for this batch");
      fd_set_tile(s->fd, (int)batch, t);
    }
    ++s->plan_gen;
  });
}

via_status via_server_set_scan_fault(via_server* s, uint32_t wait_us) {
  return guarded([&] {
    if (!s) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null handle");
    if (wait_us > 100000) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "wait_us must be at most 100000");
    std::lock_guard<std::mutex> g(s->mu);
    std::unique_lock<std::shared_mutex> plan(s->plan_mu);
    if (!s->tensor_fd()) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "this server's scan has no bounded waits (schoolbook ring)");
    VIA_CUDA(cudaStreamSynchronize(s->stream));
    s->fd.fault_wait_ns = wait_us * 1000u;
    if (wait_us == 0) {  // back to normal: forget the error word of the faulted scans
      VIA_CUDA(cudaMemsetAsync(s->fd_err.p, 0, 8, s->stream));
      VIA_CUDA(cudaStreamSynchronize(s->stream));
    }
    ++s->plan_gen;  // answer graphs captured with the other setting are re-captured
  });
}

uint64_t via_scan_tile_candidates(via_server* s, uint32_t batch, via_scan_tile* out, uint64_t cap) {
  if (!s || !s->tensor_fd() || batch == 0 || batch > 4096) return 0;
  std::vector<FdTile> c;
  try {
    c = fd_tile_candidates(s->fd, (int)batch);
  } catch (...) {
    return 0;
  }
  if (out)
    for (uint64_t i = 0; i < std::min<uint64_t>(cap, c.size()); ++i) out[i] = to_abi(c[i]);
  return c.size();
}

via_status via_server_answer_many_dev(via_server* s, const uint64_t* queries, uint64_t n_queries, uint64_t n_lwe,
                                      uint64_t* out_masks, uint64_t* out_bodies, void* stream) {
  return guarded([&] {
    if (!s || !queries || !out_masks || !out_bodies || n_queries == 0)
      throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument or empty batch");
    const via_params& p = s->prm;
    if (n_lwe != query_lwes(p))
      throw ApiError(VIA_ERR_QUERY_LENGTH_MISMATCH, "query length mismatch: expected " +
                                                        std::to_string(query_lwes(p)) + " ciphertexts, got " +
                                                        std::to_string(n_lwe));
    if (!s->cascade_eval.p) throw ApiError(VIA_ERR_SETUP_NOT_COMPLETE, "server has no public keys");
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> g(s->mu);
    ensure_batch(s, n_queries);
    VIA_CUDA(cudaMemcpyAsync(workspace_query(*s), queries, n_queries * n_lwe * lwe_len(p) * 8,
                             cudaMemcpyDeviceToDevice, st));
    answer_graph(*s, (int)n_queries, st);
    VIA_CUDA(cudaMemcpyAsync(out_masks, workspace_answer_mask(*s), n_queries * p.n2 * 8, cudaMemcpyDeviceToDevice, st));
    VIA_CUDA(cudaMemcpyAsync(out_bodies, workspace_answer_body(*s), n_queries * p.n2 * 8, cudaMemcpyDeviceToDevice, st));
  });
}

via_status via_server_answer_many(via_server* s, const uint64_t* queries, uint64_t n_queries, uint64_t n_lwe,
                                  uint64_t* out_masks, uint64_t* out_bodies) {
  return guarded([&] {
    if (!s || !queries || !out_masks || !out_bodies || n_queries == 0)
      throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument or empty batch");
    const via_params& p = s->prm;
    if (n_lwe != query_lwes(p))
      throw ApiError(VIA_ERR_QUERY_LENGTH_MISMATCH, "query length mismatch: expected " +
                                                        std::to_string(query_lwes(p)) + " ciphertexts, got " +
                                                        std::to_string(n_lwe));
    if (!s->cascade_eval.p) throw ApiError(VIA_ERR_SETUP_NOT_COMPLETE, "server has no public keys");
    std::lock_guard<std::mutex> g(s->mu);
    ensure_batch(s, n_queries);
    VIA_CUDA(cudaMemcpyAsync(workspace_query(*s), queries, n_queries * n_lwe * lwe_len(p) * 8,
                             cudaMemcpyHostToDevice, s->stream));
    answer_graph(*s, (int)n_queries, s->stream);
    VIA_CUDA(cudaMemcpyAsync(out_masks, workspace_answer_mask(*s), n_queries * p.n2 * 8, cudaMemcpyDeviceToHost,
                             s->stream));
    VIA_CUDA(cudaMemcpyAsync(out_bodies, workspace_answer_body(*s), n_queries * p.n2 * 8, cudaMemcpyDeviceToHost,
                             s->stream));
    VIA_CUDA(cudaStreamSynchronize(s->stream));
    check_device_flags(*s, s->stream);
  });
}

static void check_batch(via_server* s, uint64_t n_queries, uint64_t n_lwe) {
  const via_params& p = s->prm;
  const u64 T = (u64)via_b_batch(p);
  if (T < 2) throw ApiError(VIA_ERR_DIM_MISMATCH, "answer_batch: the server was set up for VIA-C (n_rec = n2)");
  if (n_queries != T)
    throw ApiError(VIA_ERR_DIM_MISMATCH, "answer_batch: batch.len() must equal T = n2 / n_rec = " + std::to_string(T));
  if (n_lwe != query_lwes(p))
    throw ApiError(VIA_ERR_QUERY_LENGTH_MISMATCH, "query length mismatch: expected " + std::to_string(query_lwes(p)) +
                                                      " ciphertexts, got " + std::to_string(n_lwe));
  if (!s->cascade_eval.p) throw ApiError(VIA_ERR_SETUP_NOT_COMPLETE, "server has no public keys");
}

via_status via_server_answer_batch_dev(via_server* s, const uint64_t* queries, uint64_t n_queries, uint64_t n_lwe,
                                       uint64_t* out_mask, uint64_t* out_body, void* stream) {
  return guarded([&] {
    if (!s || !queries || !out_mask || !out_body) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument");
    check_batch(s, n_queries, n_lwe);
    const via_params& p = s->prm;
    cudaStream_t st = (cudaStream_t)stream;
    (void)p;
    std::lock_guard<std::mutex> g(s->mu);
    ensure_batch(s, std::min<u64>(n_queries, VIA_B_CHUNK));
    answer_batch_device(*s, queries, out_mask, out_body, st);
  });
}

via_status via_server_answer_batch(via_server* s, const uint64_t* queries, uint64_t n_queries, uint64_t n_lwe,
                                   uint64_t* out_mask, uint64_t* out_body) {
  return guarded([&] {
    if (!s || !queries || !out_mask || !out_body) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument");
    check_batch(s, n_queries, n_lwe);
    const via_params& p = s->prm;
    std::lock_guard<std::mutex> g(s->mu);
    ensure_batch(s, std::min<u64>(n_queries, VIA_B_CHUNK));
    const size_t bytes = n_queries * n_lwe * lwe_len(p) * 8;
    DevBuf big;  // a batch larger than the workspace is uploaded whole and answered in chunks
    u64* dq = workspace_query(*s);
    if (n_queries > (u64)workspace_batch(*s)) {
      big.alloc(bytes / 8);
      dq = big.p;
    }
    VIA_CUDA(cudaMemcpyAsync(dq, queries, bytes, cudaMemcpyHostToDevice, s->stream));
    answer_batch_device(*s, dq, workspace_answer_mask(*s), workspace_answer_body(*s), s->stream);
    VIA_CUDA(cudaMemcpyAsync(out_mask, workspace_answer_mask(*s), p.n2 * 8, cudaMemcpyDeviceToHost, s->stream));
    VIA_CUDA(cudaMemcpyAsync(out_body, workspace_answer_body(*s), p.n2 * 8, cudaMemcpyDeviceToHost, s->stream));
    VIA_CUDA(cudaStreamSynchronize(s->stream));
    check_device_flags(*s, s->stream);
  });
}

uint64_t via_kernel_launches(void) { return __atomic_load_n(&g_kernel_launches, __ATOMIC_RELAXED); }

via_status via_server_answer(via_server* s, const uint64_t* query, uint64_t n_lwe, uint64_t* out_mask,
                             uint64_t* out_body) {
  return guarded([&] {
    if (!s || !query || !out_mask || !out_body) throw ApiError(VIA_ERR_INVALID_ARGUMENT, "null argument");
    const via_params& p = s->prm;
    u64 expected = query_lwes(p);
    if (n_lwe != expected)
      throw ApiError(VIA_ERR_QUERY_LENGTH_MISMATCH, "query length mismatch: expected " + std::to_string(expected) +
                                                        " ciphertexts, got " + std::to_string(n_lwe));
    if (!s->cascade_eval.p) throw ApiError(VIA_ERR_SETUP_NOT_COMPLETE, "server has no public keys");
    u64 qlen = n_lwe * lwe_len(p);
    std::lock_guard<std::mutex> g(s->mu);
    VIA_CUDA(cudaMemcpyAsync(workspace_query(*s), query, qlen * 8, cudaMemcpyHostToDevice, s->stream));
    answer_graph(*s, 1, s->stream);
    VIA_CUDA(cudaMemcpyAsync(out_mask, workspace_answer_mask(*s), p.n2 * 8, cudaMemcpyDeviceToHost, s->stream));
    VIA_CUDA(cudaMemcpyAsync(out_body, workspace_answer_body(*s), p.n2 * 8, cudaMemcpyDeviceToHost, s->stream));
    VIA_CUDA(cudaStreamSynchronize(s->stream));
    check_device_flags(*s, s->stream);
  });
}

}  // extern "C"
